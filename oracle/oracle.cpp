/*
 * oracle.cpp -- serial FP64 CPU restatement of the ADCIRC 2DDI hot path.
 *
 * TEST INFRASTRUCTURE: the checker for the CUDA library, never the product.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load it.
 *
 * Each routine follows the cited reference routine statement by statement
 * (adcirc v56.2.1, src/...).  Loop order and expression order are kept so
 * floating-point results reproduce a serial, no-FMA build of the Fortran
 * (built with -ffp-contract=off).  Branches for features the pinned
 * configuration turns off (3D, subgrid, sponge layers, weirs, condensed
 * nodes, periodic BCs, flux BCs, Manning/Chezy friction, spherical
 * coordinates) are not restated; in Cartesian coordinates (ICS=1) every
 * spherical factor (SFAC, SFCT, SFMX, ...) is exactly 1.0 and TANPHI is 0,
 * so multiplications by them are exact and are omitted.
 *
 * Parity is unpinned against the reference binary: no Fortran compiler is
 * available and the reference ships no golden vectors for this path.
 */
#include "oracle.h"

#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>

/* Thread-parallel variant for the multi-core CPU baseline only.  The
 * checker is built without ORC_THREADS: par_for is then a plain loop in
 * index order and orc_add a plain add, so its arithmetic is unchanged.
 * The threaded build (liboracle_mt.so) splits the loops into contiguous
 * chunks over std::thread workers, sums dot products per chunk and
 * scatters element contributions with atomic adds, so its sums are
 * ordered differently. */
#ifdef ORC_THREADS
#include <atomic>
#include <functional>
#include <thread>
namespace {
int orc_nthreads() {
  static int n = [] {
    const char *e = std::getenv("ORC_THREADS");
    int v = e ? std::atoi(e) : (int)std::thread::hardware_concurrency();
    return v > 0 ? v : 1;
  }();
  return n;
}
// Persistent workers released by a generation counter; the caller runs
// chunk 0 and waits for the others.
struct Pool {
  int T;
  std::vector<std::thread> th;
  std::atomic<unsigned> gen{0};
  std::atomic<int> done{0};
  std::function<void(int, int)> job;   // (thread, nthreads)
  explicit Pool(int t) : T(t) {
    for (int k = 1; k < T; ++k)
      th.emplace_back([this, k] {
        unsigned seen = 0;
        for (;;) {
          unsigned g;
          while ((g = gen.load(std::memory_order_acquire)) == seen) std::this_thread::yield();
          seen = g;
          job(k, T);
          done.fetch_add(1, std::memory_order_acq_rel);
        }
      });
    for (auto &x : th) x.detach();
  }
  void run(const std::function<void(int, int)> &f) {
    job = f;
    done.store(0, std::memory_order_relaxed);
    gen.fetch_add(1, std::memory_order_acq_rel);
    f(0, T);
    while (done.load(std::memory_order_acquire) != T - 1) std::this_thread::yield();
  }
};
Pool &pool() {
  static Pool *p = new Pool(orc_nthreads());
  return *p;
}
template <class F>
void par_for(int n, F f) {
  if (orc_nthreads() <= 1 || n < 4096) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  pool().run([&](int t, int T) {
    const int i0 = (int)((long long)n * t / T), i1 = (int)((long long)n * (t + 1) / T);
    for (int i = i0; i < i1; ++i) f(i);
  });
}
inline void orc_add(double &x, double v) { std::atomic_ref<double>(x).fetch_add(v, std::memory_order_relaxed); }
}  // namespace
#else
namespace {
template <class F>
inline void par_for(int n, F f) {
  for (int i = 0; i < n; ++i) f(i);
}
inline void orc_add(double &x, double v) { x = x + v; }
}  // namespace
#endif

namespace {

/* ------------------------------------------------------------------ */
/* ITPACK module state: common blocks /itcom1-3/ plus SAVEd locals.    */
/* ------------------------------------------------------------------ */
struct Itpack {
  int in = 0, is = 0, isym = 0, itmax = 0, level = -1, nout = 6;
  bool adapt = false, betadt = false, caseii = false, halt = false, partad = false;
  double bdelnm = 0, betab = 0, cme = 0, delnnm = 0, delsnm = 0, ff = 0,
         gamma = 0, omega = 0, qa = 0, qt = 0, rho = 0, rrr = 0, sige = 0,
         sme = 0, specr = 0, spr = 0, srelpr = DBL_EPSILON, stptst = 0,
         udnm = 0, zeta = 0;
  /* itjcg SAVEd locals (itpackv.F:459-604, `save`) */
  bool q1 = false;
  double gamold = 0, rhoold = 0;
  /* chgcon SAVEd locals (itpackv.F:893-1027, `save`) */
  double cmold = 0;
  int chg_ier = 0;
};

Itpack g_itp; /* process-global, like the Fortran common blocks */

/* sdot, itpackv.F:2828-2845: plain sequential sum. */
double sdot(int n, const double *x, const double *y) {
  double d = 0.0;
#ifdef ORC_THREADS
  if (orc_nthreads() > 1 && n >= 4096) {
    std::vector<double> part(orc_nthreads(), 0.0);
    pool().run([&](int t, int T) {
      const int i0 = (int)((long long)n * t / T), i1 = (int)((long long)n * (t + 1) / T);
      double s = 0.0;
      for (int i = i0; i < i1; ++i) s = s + x[i] * y[i];
      part[t] = s;
    });
    for (double v : part) d = d + v;
    return d;
  }
#endif
  for (int i = 0; i < n; ++i) d = d + x[i] * y[i];
  return d;
}

/* pjac, itpackv.F:1932-1967: rhs(i) -= coef(i,j)*u(jcoef(i,j)), j=2..maxnz. */
void pjac(int n, int ndim, int maxnz, const int *jcoef, const double *coef,
          const double *u, double *rhs) {
  for (int j = 1; j < maxnz; ++j)
    par_for(n, [&](int i) {
      rhs[i] = rhs[i] - coef[i + (size_t)ndim * j] * u[jcoef[i + (size_t)ndim * j] - 1];
    });
}

/* pmult, itpackv.F:1970-2005 (c = b - sum_j coef(:,j)*b(jcoef(:,j))). */
void pmult(int n, int ndim, int maxnz, const int *jcoef, const double *coef,
           const double *b, double *c) {
  for (int i = 0; i < n; ++i) c[i] = b[i];
  for (int j = 1; j < maxnz; ++j)
    par_for(n, [&](int i) {
      c[i] = c[i] - coef[i + (size_t)ndim * j] * b[jcoef[i + (size_t)ndim * j] - 1];
    });
}

/* determ, itpackv.F:1029-1068: characteristic polynomial of tri at xlmda. */
double determ(int ldt, int n, const double *tri, double *wk1, double *wk2, double xlmda) {
  /* tri(ldt,2): tri(i,1)=tri[i-1], tri(i,2)=tri[ldt+i-1] */
  for (int i = 1; i <= n; ++i) wk1[i - 1] = tri[i - 1] - xlmda;
  wk2[n - 1] = wk1[n - 1];
  wk2[n - 2] = wk1[n - 2] * wk2[n - 1] + tri[ldt + n - 1];
  if (n != 2) {
    for (int l = n - 2; l >= 1; --l)
      wk2[l - 1] = wk1[l - 1] * wk2[l] + tri[ldt + l] * wk2[l + 1];
  }
  return wk2[0];
}

/* zbrent, itpackv.F:2521-2781 (modified IMSL Brent root finder). */
void zbrent(int n, double *tri, double eps, int nsig, double &a, double &b,
            int &maxfn, int &ier) {
  Itpack &c_ = g_itp;
  double c = 0, d = 0, e = 0, p, q, r, s, fa, fb, fc, tol, rm, rone, temp;
  ier = 0;
  const int ib3 = 2 * c_.itmax;   /* tri(ib3) = tri(2*itmax+1) */
  const int ib4 = 3 * c_.itmax;
  double t = std::pow(10.0, -nsig);
  int ic = 2;
  fa = determ(c_.itmax, n, tri, tri + ib3, tri + ib4, a);
  fb = determ(c_.itmax, n, tri, tri + ib3, tri + ib4, b);
  s = b;
  if ((fa > 0.0 && fb > 0.0) || (fa < 0.0 && fb < 0.0)) {
    ier = 502;
    maxfn = ic;
    return;
  }
L10:
  c = a;
  fc = fa;
  d = b - c;
  e = d;
L20:
  if (!(std::fabs(fc) >= std::fabs(fb))) {
    a = b; b = c; c = a;
    fa = fb; fb = fc; fc = fa;
  }
  tol = t * std::max(std::fabs(b), 0.1);
  rm = (c - b) * 0.5;
  if (std::fabs(fb) <= eps) goto L80;
  if (std::fabs(c - b) <= tol) goto L80;
  if (ic >= maxfn) goto L90;
  if (std::fabs(e) < tol) goto L60;
  if (std::fabs(fa) <= std::fabs(fb)) goto L60;
  s = fb / fa;
  if (a != c) goto L40;
  p = (c - b) * s;
  q = 1.0 - s;
  goto L50;
L40:
  q = fa / fc;
  r = fb / fc;
  rone = r - 1.0;
  p = s * ((c - b) * q * (q - r) - (b - a) * rone);
  q = (q - 1.0) * rone * (s - 1.0);
L50:
  if (p > 0.0) q = -q;
  if (p < 0.0) p = -p;
  s = e;
  e = d;
  if (p + p >= 3.0 * rm * q) goto L60;
  if (p + p >= std::fabs(s * q)) goto L60;
  d = p / q;
  goto L70;
L60:
  e = rm;
  d = e;
L70:
  a = b;
  fa = fb;
  temp = d;
  if (std::fabs(temp) <= 0.5 * tol) temp = std::copysign(0.5 * tol, rm);
  b = b + temp;
  s = b;
  fb = determ(c_.itmax, n, tri, tri + ib3, tri + ib4, s);
  ic = ic + 1;
  if (fb == 0.0 || fc == 0.0) goto L20;
  if ((fb > 0.0 && fc < 0.0) || (fb < 0.0 && fc > 0.0)) goto L20;
  goto L10;
L80:
  a = c;
  maxfn = ic;
  return;
L90:
  ier = 501;
  a = c;
  maxfn = ic;
}

/* eigvss, itpackv.F:1361-1399. */
double eigvss(int n, double *tri, double start, double zeta, int itmax, int &ier) {
  int itmp = (int)(-std::log10(std::fabs(zeta)));
  int nsig = std::max(itmp, 4);
  int maxfn = std::max(itmax, 50);
  double eps = 0.0, a = start, b = 1.0;
  zbrent(n, tri, eps, nsig, a, b, maxfn, ier);
  return b;
}

/* chgcon, itpackv.F:893-1027, jacobi case (ibmth = 1). */
void chgcon(double *tri, double gamold, double rhoold) {
  Itpack &c = g_itp;
  const int ldt = c.itmax;
  double start = c.cme, end1 = 0.0;
  int ip = c.in;
  if (ip >= 2) goto L60;
  if (ip == 1) goto L50;
  end1 = 0.0;
  c.cmold = 0.0;
  goto L110;
L50:
  end1 = 1.0 - 1.0 / c.gamma;
  tri[0] = end1;
  tri[ldt] = 0.0;
  goto L110;
L60:
  if (std::fabs(start - c.cmold) <= c.zeta * start) goto L120;
  c.cmold = start;
  tri[ip - 1] = 1.0 - 1.0 / c.gamma;
  tri[ldt + ip - 1] = (1.0 - c.rho) / (c.rho * rhoold * c.gamma * gamold);
  if (c.isym != 0) {
    /* eigvns/eqrt1s (mixed-sign diagonals) is not restated: report it. */
    c.chg_ier = 903;
  } else {
    end1 = eigvss(ip, tri, start, c.zeta, c.itmax, c.chg_ier);
  }
  if (c.chg_ier != 0) goto L130;
L110:
  c.cme = end1;
  return;
L120:
  c.adapt = false;
  c.partad = false;
  return;
L130:
  c.adapt = false;
  c.partad = false;
}

/* pstop_nrms, itpackv.F:809-890 (iflag = 1). */
void pstop_nrms(double unrm, double dnrm, double ccon, bool &q1) {
  Itpack &c = g_itp;
  double con = ccon, uold, tr, tl;
  c.halt = false;
  if (c.in < 1) {
    q1 = false;
    c.udnm = 1.0;
    c.stptst = 1000.0;
  }
  if (!q1 && !((c.in > 5) && (c.in % 5 != 0))) {
    uold = c.udnm;
    c.udnm = unrm;
    if (c.udnm == 0.0) c.udnm = 1.0;
    if ((c.in > 5) && (std::fabs(c.udnm - uold) <= c.udnm * c.zeta)) q1 = true;
  }
  tr = std::sqrt(c.udnm);
  tl = 1.0;
  if (con != 1.0) {
    tl = std::sqrt(dnrm);
    tr = tr * (1.0 - con);
  }
  c.stptst = tl / tr;
  if (tl >= tr * c.zeta) return;
  c.halt = true;
}

/* parcon, itpackv.F:1774-1851 (jacobi case). */
void parcon(double dtnrm, double &c1, double &c2, double &c3, double &c4,
            double &gamold, double &rhotmp) {
  Itpack &c = g_itp;
  int ip = c.in - c.is;
  double rhoold = c.rho;
  gamold = c.gamma;
  c.gamma = 1.0 / (1.0 - dtnrm / c.delnnm);
  c.rho = 1.0;
  if (ip != 0) c.rho = 1.0 / (1.0 - c.gamma * c.delnnm / (gamold * c.delsnm * rhoold));
  c.delsnm = c.delnnm;
  rhotmp = rhoold;
  c1 = c.rho * c.gamma;
  c2 = c.rho;
  c3 = 1.0 - c.rho;
  c4 = c.rho * (1.0 - c.gamma);
}

/* itjcg, itpackv.F:459-604 (serial build: sdot for the norms). */
void itjcg(int n, int ndim, int maxnz, const int *jcoef, const double *coef,
           const double *u, double *u1, const double *d, double *d1, double *dtwd,
           double *tri) {
  Itpack &c = g_itp;
  double dtnrm, unorm, c1, c2, c3, c4;
  if (c.adapt) chgcon(tri, c.gamold, c.rhoold);
  for (int i = 0; i < n; ++i) dtwd[i] = 0.0;
  pjac(n, ndim, maxnz, jcoef, coef, d, dtwd);
  if (c.q1 || ((c.in > 5) && (c.in % 5 != 0))) {
    c.delnnm = sdot(n, d, d);
    dtnrm = sdot(n, d, dtwd);
    unorm = 1.0;
  } else {
    c.delnnm = sdot(n, d, d);
    dtnrm = sdot(n, d, dtwd);
    unorm = sdot(n, u, u);
  }
  double dnrm = c.delnnm;
  pstop_nrms(unorm, dnrm, c.cme, c.q1);
  if (c.halt) return;
  parcon(dtnrm, c1, c2, c3, c4, c.gamold, c.rhoold);
  par_for(n, [&](int i) {
    u1[i] = c1 * d[i] + c2 * u[i] + c3 * u1[i];
    d1[i] = c1 * dtwd[i] + c4 * d[i] + c3 * d1[i];
  });
}

/* scal, itpackv.F:2281-2421. */
void scal(int n, int ndim, int maxnz, int *jcoef, double *coef, double *rhs,
          double *u, double *work, int &ier) {
  Itpack &c = g_itp;
  int nsgncg = 0;
  ier = 0;
  if (n <= 0) return;
  for (int i = 1; i <= n; ++i) {
    int *jr = jcoef + (i - 1);
    double *cr = coef + (i - 1);
    if (jr[0] != i) {
      if (maxnz < 2) { ier = 402; return; }
      for (int j = 2; j <= maxnz; ++j) {
        if (jr[(size_t)ndim * (j - 1)] == i) {
          double save = cr[(size_t)ndim * (j - 1)];
          cr[(size_t)ndim * (j - 1)] = cr[0];
          jr[(size_t)ndim * (j - 1)] = jr[0];
          cr[0] = save;
          jr[0] = i;
        }
      }
    }
    if (cr[0] < 0.0) {
      for (int j = 1; j <= maxnz; ++j) cr[(size_t)ndim * (j - 1)] = -cr[(size_t)ndim * (j - 1)];
      rhs[i - 1] = -rhs[i - 1];
      nsgncg = nsgncg + 1;
    } else if (cr[0] == 0.0) {
      ier = 401;
      return;
    }
  }
  if (maxnz >= 2) {
    for (int j = 2; j <= maxnz; ++j)
      for (int i = 1; i <= n; ++i)
        if (jcoef[(i - 1) + (size_t)ndim * (j - 1)] <= 0) jcoef[(i - 1) + (size_t)ndim * (j - 1)] = i;
  }
  for (int i = 0; i < n; ++i) work[i] = std::sqrt(coef[i]);
  for (int i = 0; i < n; ++i) u[i] = u[i] * work[i];
  for (int i = 0; i < n; ++i) work[i] = 1.0 / work[i];
  for (int i = 0; i < n; ++i) coef[i] = work[i];
  for (int i = 0; i < n; ++i) rhs[i] = rhs[i] * work[i];
  if (maxnz < 2) return;
  for (int j = 2; j <= maxnz; ++j)
    for (int i = 0; i < n; ++i) {
      size_t k = i + (size_t)ndim * (j - 1);
      coef[k] = coef[k] * work[i] * work[jcoef[k] - 1];
    }
  if (nsgncg > 0 && nsgncg < n) c.isym = 1;
}

/* unscal, itpackv.F:2424-2479. */
void unscal(int n, int ndim, int maxnz, int *jcoef, double *coef, double *rhs,
            double *u, double *work) {
  for (int i = 0; i < n; ++i) work[i] = coef[i];
  for (int i = 0; i < n; ++i) u[i] = u[i] * work[i];
  for (int i = 0; i < n; ++i) work[i] = 1.0 / work[i];
  for (int i = 0; i < n; ++i) rhs[i] = rhs[i] * work[i];
  if (maxnz >= 2) {
    for (int j = 2; j <= maxnz; ++j)
      for (int i = 0; i < n; ++i) {
        size_t k = i + (size_t)ndim * (j - 1);
        coef[k] = coef[k] * work[i] * work[jcoef[k] - 1];
      }
    for (int j = 2; j <= maxnz; ++j)
      for (int i = 1; i <= n; ++i) {
        size_t k = (i - 1) + (size_t)ndim * (j - 1);
        if (jcoef[k] == i) jcoef[k] = 0;
      }
  }
  for (int i = 0; i < n; ++i) coef[i] = work[i] * work[i];
}

/* peror, itpackv.F:607-720 (digit1/digit2 diagnostics only). */
void peror(int n, int ndim, int maxnz, const int *jcoef, const double *coef,
           const double *rhs, const double *u, double *work, double &digit1,
           double &digit2) {
  Itpack &c = g_itp;
  digit1 = 0.0;
  digit2 = 0.0;
  if (n <= 0) return;
  digit1 = -std::log10(std::fabs(c.srelpr));
  if (c.stptst > 0.0) digit1 = -std::log10(std::fabs(c.stptst));
  for (int i = 0; i < n; ++i) work[i] = rhs[i] / coef[i];
  double bnrm = sdot(n, work, work);
  if (bnrm == 0.0) { digit2 = -std::log10(std::fabs(c.srelpr)); return; }
  std::vector<double> tmp(n);
  pmult(n, ndim, maxnz, jcoef, coef, u, tmp.data());
  for (int i = 0; i < n; ++i) work[i] = (rhs[i] - tmp[i]) / coef[i];
  double rnrm = sdot(n, work, work);
  double temp = rnrm / bnrm;
  if (temp == 0.0) { digit2 = -std::log10(std::fabs(c.srelpr)); return; }
  digit2 = -std::log10(std::fabs(temp)) / 2.0;
}

/* echall (icall = 1), itpackv.F:1172-1256. */
void echall(const int *iparm, const double *rparm) {
  Itpack &c = g_itp;
  c.zeta = rparm[0];
  c.cme = rparm[1];
  c.sme = rparm[2];
  c.ff = rparm[3];
  c.omega = rparm[4];
  c.specr = rparm[5];
  c.betab = rparm[6];
  c.itmax = iparm[0];
  c.level = iparm[1];
  c.isym = iparm[4];
  c.adapt = false;
  c.partad = false;
  c.betadt = false;
  if (iparm[5] == 1 || iparm[5] == 3) c.adapt = true;
  if (iparm[5] == 1) c.betadt = true;
  if (iparm[5] == 2) c.partad = true;
  c.caseii = (iparm[6] == 2);
  if (c.caseii) c.sme = -c.cme;
  if (!c.caseii && c.sme == 0.0) c.sme = -1.0;
  c.spr = c.sme;
  c.in = 0;
  c.is = 0;
  c.halt = false;
  c.bdelnm = c.delnnm = c.delsnm = c.gamma = c.qa = c.qt = c.rho = c.rrr =
      c.sige = c.stptst = c.udnm = 0.0;
}

void jcg_impl(int n, int ndim, int maxnz, int *jcoef, double *coef, double *rhs,
              double *u, int *iwksp, int nw, double *wksp, int *iparm,
              double *rparm, int &ier) {
  (void)iwksp;
  Itpack &c = g_itp;
  ier = 0;
  c.level = iparm[1];
  c.nout = iparm[3];
  if (iparm[0] <= 0) return;
  echall(iparm, rparm);
  double temp = 512.0 * c.srelpr;
  if (c.zeta < temp) c.zeta = temp;
  double digit1 = rparm[10], digit2 = rparm[11];
  if (n <= 0) { ier = 11; return; }
  scal(n, ndim, maxnz, jcoef, coef, rhs, u, wksp, ier);
  if (ier != 0) return;
  /* iparm(10) (sbelm) and iparm(9) >= -1 (red-black) are not restated:
   * the GWCE caller uses the dfault values 0 and -2. */
  const int ib1 = 0, ib2 = n, ib3 = 2 * n, ib4 = 3 * n, ib5 = 4 * n;
  int nb = iparm[8];
  iparm[7] = 4 * n + 4 * c.itmax;
  if (nw < iparm[7]) {
    ier = 12;
  } else {
    for (int i = 0; i < nw; ++i) wksp[i] = 0.0;
    for (int i = 0; i < n; ++i) wksp[ib2 + i] = rhs[i];
    pjac(n, ndim, maxnz, jcoef, coef, u, wksp + ib2);
    for (int i = 0; i < n; ++i) wksp[n + i] = wksp[n + i] - u[i];
    int itmax1 = c.itmax + 1;
    bool converged = false;
    for (int loop = 1; loop <= itmax1; ++loop) {
      c.in = loop - 1;
      if (c.in % 2 == 1) {
        itjcg(n, ndim, maxnz, jcoef, coef, wksp + ib1, u, wksp + ib3, wksp + ib2,
              wksp + ib4, wksp + ib5);
      } else {
        itjcg(n, ndim, maxnz, jcoef, coef, u, wksp + ib1, wksp + ib2, wksp + ib3,
              wksp + ib4, wksp + ib5);
      }
      if (c.halt) { converged = true; break; }
    }
    if (!converged) {
      ier = 13;
      if (iparm[2] == 0) rparm[0] = c.stptst;
    }
    if (c.in % 2 == 1)
      for (int i = 0; i < n; ++i) u[i] = wksp[i];
  }
  int idgts = iparm[11];
  if (idgts >= 0) {
    peror(n, ndim, maxnz, jcoef, coef, rhs, u, wksp, digit1, digit2);
  }
  unscal(n, ndim, maxnz, jcoef, coef, rhs, u, wksp);
  iparm[7] = iparm[7] - 4 * (c.itmax - c.in);
  if (iparm[2] != 0) return;
  iparm[0] = c.in;
  iparm[8] = nb;
  rparm[1] = c.cme;
  rparm[2] = c.sme;
  rparm[10] = digit1;
  rparm[11] = digit2;
}

/* ------------------------------------------------------------------ */
/* Model oracle                                                        */
/* ------------------------------------------------------------------ */

inline int NM(const orc_arrays_t *a, int ie, int k) { /* 0-based ie,k -> 0-based node */
  return a->nm[ie + (size_t)a->ne * k] - 1;
}

} /* namespace */

struct orc_model {
  orc_params_t p;
  orc_arrays_t *a;
  /* NWS = 8 vortex: track, options and GetHollandStormData's module state
   * (bestTrackCounter, WTRATIO; nws08.F90:68, 114) */
  /* specified normal flux: NFLUXF, the constituents and QN0/QN1/QN2 (NVEL) */
  int nfluxf = 0, flux_on = 0, nffr = 0;
  int nfluxrbc = 0;   /* radiation (IBTYPE 30) entries, mesh.F:2045 */
  int nfluxgbc = 0;   /* zero normal velocity gradient (IBTYPE 40) entries, mesh.F:2072 */
  int nfluxb = 0;     /* external barrier (IBTYPE 3/13/23) entries, mesh.F:1913 */
  int nfluxib = 0;    /* internal barrier (IBTYPE 4/24/5/25) entries, mesh.F:1919, 1924 */
  int nfluxibp = 0;   /* barriers with pipes (IBTYPE 5/25), mesh.F:1925 */
  std::vector<int> nib, nibcnt;   /* NIBNODECODE, NIBCNT (NP) */
  /* river radiation (IBTYPE 52): FluxSettlingIT, EtaDisc_Fill and
   * EtaDisc/ElevDisc at the boundary entries (timestep.F:183, 243-245) */
  int flux_settling_it = 0, etadisc_fill = 1;
  std::vector<double> elevdisc, etadisc_b;
  std::vector<double> famig, fper, fff, fface, qnam, qnph, qn0, qn1, qn2;
  /* coupled flux/radiation (IBTYPE 32): ENAM/ENPH and EN0/EN1/EN2 (NVEL) */
  std::vector<double> enam, enph, en0, en1, en2;
  /* fort.19 (NPEBC) and fort.20 (NFFR <= 0) series as the reference holds
   * them: the two records in use (ESBIN1/ESBIN2, QNIN1/QNIN2, ENIN1/ENIN2),
   * their times, and the next record of the file to read */
  int npebc = 0, fser_on = 0, series_err = 0;
  double etiminc = 0, etime1 = 0, etime2 = 0, ftiminc = 0, qtime1 = 0, qtime2 = 0;
  std::vector<double> e19, q20, e20;   /* the files' records */
  int e19_nrec = 0, q20_nrec = 0, e19_next = 0, q20_next = 0;
  std::vector<double> esbin1, esbin2, qnin1, qnin2, enin1, enin2;
  int vortex_on = 0;
  orc_vortex_t vpar;
  std::vector<orc_vortex_fix_t> vfix;
  int vcounter = 0;
  double vwtratio = 1.0;
  int iparm[12];
  double rparm[12];
  int ncchange;
  double ep;
  std::vector<int> iwksp;
  std::vector<double> wksp;
  std::vector<double> tk_tmp;
  int nw;
};

extern "C" {

void orc_dfault(int *iparm, double *rparm) {
  /* dfault, itpackv.F:1070-1170 */
  g_itp.srelpr = DBL_EPSILON;
  iparm[0] = 100; iparm[1] = -1; iparm[2] = 0; iparm[3] = 6; iparm[4] = 0;
  iparm[5] = 1; iparm[6] = 1; iparm[7] = 0; iparm[8] = -2; iparm[9] = 0;
  iparm[10] = 0; iparm[11] = 3;
  rparm[0] = 5.0e-6; rparm[1] = 0.0; rparm[2] = 0.0; rparm[3] = 0.75;
  rparm[4] = 1.0; rparm[5] = 0.0; rparm[6] = 0.25; rparm[7] = 128.0 * g_itp.srelpr;
  rparm[8] = 0.0; rparm[9] = 0.0; rparm[10] = 0.0; rparm[11] = 0.0;
}

void orc_itpack_reset(void) { g_itp = Itpack(); }

void orc_jcg(const int *n, const int *ndim, const int *maxnz, int *jcoef,
             double *coef, double *rhs, double *u, int *iwksp, const int *nw,
             double *wksp, int *iparm, double *rparm, int *ier) {
  int e = 0;
  jcg_impl(*n, *ndim, *maxnz, jcoef, coef, rhs, u, iwksp, *nw, wksp, iparm, rparm, e);
  *ier = e;
}

orc_model *orc_model_create(const orc_params_t *p, orc_arrays_t *a) {
  orc_model *m = new orc_model();
  m->p = *p;
  m->a = a;
  orc_itpack_reset();
  /* initGWCE, gwce.F:123-157 */
  orc_dfault(m->iparm, m->rparm);
  m->iparm[0] = p->itmax;
  m->iparm[1] = p->isldia;
  m->iparm[3] = 16;
  m->rparm[0] = p->convcr;
  m->nw = 4 * a->np + 4 * p->itmax;
  m->iwksp.assign(3 * (size_t)a->np, 0);
  /* NFLUXF, mesh.F:1907 etc.: any specified-flux segment */
  for (int I = 0; I < a->nvel; ++I) {
    const int lb = a->lbcodei[I];
    if (lb == 2 || lb == 12 || lb == 22 || lb == 32 || lb == 52) m->nfluxf = 1;
    if (lb == 30 || lb == 32) m->nfluxrbc = 1;   /* mesh.F:2044-2045, 2056-2058 */
    if (lb == 40 || lb == 41) m->nfluxgbc = 1;
    if (lb == 3 || lb == 13 || lb == 23) m->nfluxb = 1;
    if (lb == 4 || lb == 24 || lb == 5 || lb == 25) m->nfluxib = 1;
    if (lb == 5 || lb == 25) m->nfluxibp = 1;
  }
  m->nib.assign(a->np, 0);
  m->nibcnt.assign(a->np, 0);
  /* EtaDisc at river-radiation nodes from the cold-start ETA2, cstart.F:1186-1191 */
  m->elevdisc.assign(std::max(a->nvel, 1), 0.0);
  m->etadisc_b.assign(std::max(a->nvel, 1), 0.0);
  for (int I = 0; I < a->nvel; ++I)
    if (a->lbcodei[I] == 52) m->etadisc_b[I] = a->eta2[a->nbv[I] - 1];
  m->qn0.assign(std::max(a->nvel, 1), 0.0);
  m->qn1 = m->qn0;
  m->qn2 = m->qn0;
  m->en0 = m->qn0;
  m->en1 = m->qn0;
  m->en2 = m->qn0;
  m->wksp.assign((size_t)4 * a->np + 400 + 4 * (size_t)p->itmax, 0.0);
  m->tk_tmp.assign(a->np, 0.0);
  m->ncchange = 1; /* adcirc.F:404 */
  m->ep = 0.0;
  return m;
}

void orc_model_destroy(orc_model *m) { delete m; }
void orc_model_set_ncchange(orc_model *m, int v) { m->ncchange = v; }
int orc_model_get_ncchange(const orc_model *m) { return m->ncchange; }
double orc_model_get_zeta(const orc_model *m) { return m->rparm[0]; }

/* TIMESTEP glue, timestep.F:231-237, 375-416, 578-592. */
int orc_model_shift_friction(orc_model *m, const orc_step_t *s) {
  orc_arrays_t *a = m->a;
  const orc_params_t &p = m->p;
  const int np = a->np;
  if (s->it == 1) {
    for (int i = 0; i < np; ++i) {
      a->h2[i] = a->dp[i] + p.ifnlfa * a->eta2[i];
      a->h1[i] = a->h2[i];
    }
  }
  for (int i = 0; i < np; ++i) {
    a->qx1[i] = a->qx2[i];
    a->qy1[i] = a->qy2[i];
    a->uu1[i] = a->uu2[i];
    a->vv1[i] = a->vv2[i];
    a->gwce_lv[i] = 0.0;
    a->mom_lv_x[i] = 0.0;
    a->mom_lv_y[i] = 0.0;
    if (p.nws != 0) {
      a->wsx1[i] = a->wsx2[i];
      a->wsx2[i] = 0.0;
      a->wsy1[i] = a->wsy2[i];
      a->wsy2[i] = 0.0;
      a->pr1[i] = a->pr2[i];
      a->pr2[i] = p.prbckgrnd_mh2o;
    } else {
      a->pr2[i] = p.prbckgrnd_mh2o;
    }
  }
  /* Apply2DBottomFriction, nodalattr.F:2399-2413 */
  const double tkcap = 2.0 / p.dt;
  for (int i = 0; i < np; ++i) {
    double uv1 = std::sqrt(a->uu1[i] * a->uu1[i] + a->vv1[i] * a->vv1[i]);
    double h1 = a->dp[i] + p.ifnlfa * a->eta2[i];
    double hyb = p.ifhybf * std::pow(1.0 + std::pow(p.hbreak / h1, p.ftheta), p.fgamma / p.ftheta);
    double v = a->fric[i] * (p.iflinbf + (uv1 / h1) * (p.ifnlbf + hyb));
    a->tk[i] = std::min(v, tkcap);
  }
  /* Apply2DInternalWaveDrag default copy, nodalattr.F:2700-2704 */
  for (int i = 0; i < np; ++i) {
    a->tkm[3 * (size_t)i + 0] = a->tk[i];
    a->tkm[3 * (size_t)i + 1] = a->tk[i];
    a->tkm[3 * (size_t)i + 2] = 0.0;
  }
  /* shift of the specified normal flux, timestep.F:606-613 */
  for (int I = 0; I < a->nvel; ++I) {
    m->qn0[I] = m->qn1[I];
    m->qn1[I] = m->qn2[I];
    m->qn2[I] = 0.0;
    m->en0[I] = m->en1[I];
    m->en1[I] = m->en2[I];
    m->en2[I] = 0.0;
  }
  return 0;
}

int orc_model_set_flux(orc_model *m, const orc_flux_t *f) {
  if (!f || f->nffr < 1 || !m->nfluxf) return 1;
  const int nf = f->nffr, nv = m->a->nvel;
  m->nffr = nf;
  m->famig.assign(f->famig, f->famig + nf);
  m->fper.assign(f->fper, f->fper + nf);
  m->fff.assign(f->fff, f->fff + nf);
  m->fface.assign(f->fface, f->fface + nf);
  m->qnam.assign(f->qnam, f->qnam + (size_t)nf * nv);
  m->qnph.assign(f->qnph, f->qnph + (size_t)nf * nv);
  if (f->enam && f->enph) {
    m->enam.assign(f->enam, f->enam + (size_t)nf * nv);
    m->enph.assign(f->enph, f->enph + (size_t)nf * nv);
  } else {
    m->enam.assign((size_t)nf * nv, 0.0);
    m->enph.assign((size_t)nf * nv, 0.0);
  }
  m->flux_settling_it = f->flux_settling_it;
  m->flux_on = 1;
  return 0;
}

int orc_model_set_elev_series(orc_model *m, const orc_series_t *s) {
  const int neta = m->a->neta;
  if (!s || s->nrec < 2 || !s->values || !(s->interval > 0.0) || neta < 1) return 1;
  m->e19.assign(s->values, s->values + (size_t)s->nrec * neta);
  m->e19_nrec = s->nrec;
  /* cstart.F:207-216: ETIMINC, two records, ETIME1 = STATIM*86400 */
  m->etiminc = s->interval;
  m->esbin1.assign(m->e19.begin(), m->e19.begin() + neta);
  m->esbin2.assign(m->e19.begin() + neta, m->e19.begin() + 2 * (size_t)neta);
  m->e19_next = 2;
  m->etime1 = s->start_time;
  m->etime2 = m->etime1 + m->etiminc;
  m->npebc = 1;
  return 0;
}

int orc_model_set_flux_series(orc_model *m, const orc_series_t *s) {
  const int nv = m->a->nvel;
  if (!s || s->nrec < 2 || !s->values || !(s->interval > 0.0) || !m->nfluxf) return 1;
  m->q20.assign(s->values, s->values + (size_t)s->nrec * nv);
  if (s->values2)
    m->e20.assign(s->values2, s->values2 + (size_t)s->nrec * nv);
  else
    m->e20.assign((size_t)s->nrec * nv, 0.0);
  m->q20_nrec = s->nrec;
  /* cstart.F:227-256: QNIN1 = QNIN2 = 0, then two records at the flux entries */
  m->ftiminc = s->interval;
  m->qnin1.assign(nv, 0.0);
  m->qnin2.assign(nv, 0.0);
  m->enin1.assign(nv, 0.0);
  m->enin2.assign(nv, 0.0);
  const orc_arrays_t *a = m->a;
  for (int J = 0; J < nv; ++J) {
    const int lb = a->lbcodei[J];
    if (lb == 2 || lb == 12 || lb == 22 || lb == 32) {
      m->qnin1[J] = m->q20[J];
      m->qnin2[J] = m->q20[(size_t)nv + J];
    }
    if (lb == 32) {
      m->enin1[J] = m->e20[J];
      m->enin2[J] = m->e20[(size_t)nv + J];
    }
  }
  m->q20_next = 2;
  m->qtime1 = s->start_time;
  m->qtime2 = m->qtime1 + m->ftiminc;
  m->flux_settling_it = s->flux_settling_it;
  m->fser_on = 1;
  m->flux_on = 0;
  return 0;
}

/* periodic specified normal flux, timestep.F:861-880 (ICS = 1: no rotation),
 * the discharge elevation of river-radiation entries, :906-926, then the
 * discharge at radiation entries, timestep.F:932-940 */
static void orc_model_flux(orc_model *m, const orc_step_t *s) {
  orc_arrays_t *a = m->a;
  const double G = m->p.g;
  if (m->nfluxf && m->flux_on) {
    for (int J = 0; J < m->nffr; ++J) {
      int NCYC = 0;
      if (m->fper[J] != 0.0) NCYC = (int)(s->timeh / m->fper[J]);
      const double ARGJ = m->famig[J] * (s->timeh - NCYC * m->fper[J]) + m->fface[J];
      const double RFF = m->fff[J] * s->rampextflux;
      for (int I = 0; I < a->nvel; ++I) {
        const int lb = a->lbcodei[I];
        if (lb == 2 || lb == 12 || lb == 22 || lb == 52 || lb == 32)
          m->qn2[I] = m->qn2[I] + m->qnam[J + (size_t)m->nffr * I] * RFF *
                                      std::cos(ARGJ - m->qnph[J + (size_t)m->nffr * I]);
        if (lb == 32)
          m->en2[I] = m->en2[I] + m->enam[J + (size_t)m->nffr * I] * RFF *
                                      std::cos(ARGJ - m->enph[J + (size_t)m->nffr * I]);
      }
    }
  } else if (m->nfluxf && m->fser_on) {
    /* non-periodic flux, timestep.F:882-903 */
    if (s->timeloc > m->qtime2) {
      m->qtime1 = m->qtime2;
      m->qtime2 = m->qtime2 + m->ftiminc;
      if (m->q20_next >= m->q20_nrec) {   /* the reference's READ hits the end of fort.20 */
        m->series_err = 1;
      } else {
        const size_t r = (size_t)m->q20_next++ * a->nvel;
        for (int J = 0; J < a->nvel; ++J) {
          const int lb = a->lbcodei[J];
          if (lb == 2 || lb == 12 || lb == 22) {
            m->qnin1[J] = m->qnin2[J];
            m->qnin2[J] = m->q20[r + J];
          } else if (lb == 32) {
            m->qnin1[J] = m->qnin2[J];
            m->enin1[J] = m->enin2[J];
            m->qnin2[J] = m->q20[r + J];
            m->enin2[J] = m->e20[r + J];
          }
        }
      }
    }
    const double QTRATIO = (s->timeloc - m->qtime1) / m->ftiminc;
    for (int I = 0; I < a->nvel; ++I) {
      m->qn2[I] = s->rampextflux * (m->qnin1[I] + QTRATIO * (m->qnin2[I] - m->qnin1[I]));
      m->en2[I] = s->rampextflux * (m->enin1[I] + QTRATIO * (m->enin2[I] - m->enin1[I]));
    }
  }
  if (m->nfluxf) {
    if (s->it == m->flux_settling_it) {
      m->etadisc_fill = 0;
      for (int I = 0; I < a->nvel; ++I)
        if (a->lbcodei[I] == 52) {
          const int NNBB = a->nbv[I] - 1;
          m->etadisc_b[I] = a->eta2[NNBB];
          m->elevdisc[I] = a->eta2[NNBB];
        }
    } else if (m->etadisc_fill && s->it > m->flux_settling_it) {
      m->etadisc_fill = 0;
      for (int I = 0; I < a->nvel; ++I)
        if (a->lbcodei[I] == 52) m->elevdisc[I] = m->etadisc_b[I];
    }
  }
  if (m->nfluxrbc) {
    for (int I = 0; I < a->nvel; ++I) {
      if (a->lbcodei[I] != 30) continue;
      const int NNBB = a->nbv[I] - 1;
      const double UN1 = a->uu1[NNBB] * a->csii[I] + a->vv1[NNBB] * a->siii[I];
      m->qn1[I] = a->h2[NNBB] * UN1;
    }
  }
  /* supercritical outflow over external barriers, timestep.F:967-975 and
   * COMPUTE_EXTERNAL_BOUNDARY_FLUX (weir_boundary.F90:1727-1763; BARMIN
   * 0.04 m, no time-varying crest) */
  if (m->nfluxb) {
    for (int I = 0; I < a->nvel; ++I) {
      const int lb = a->lbcodei[I];
      if (lb != 3 && lb != 13 && lb != 23) continue;
      const int NNBB = a->nbv[I] - 1;
      const double RBARWL = 2.0 * (a->eta2[NNBB] - a->barlanht[I]) / 3.0;
      if (RBARWL > 0.04)
        m->qn2[I] = -s->rampintflux * a->barlancfsp[I] * RBARWL * std::sqrt(RBARWL * G);
      else
        m->qn2[I] = 0.0;
    }
  }
  /* flow between the faces of internal barriers, timestep.F:1003-1026 and
   * COMPUTE_INTERNAL_BOUNDARY_FLUX (weir_boundary.F90:1775-1942; default
   * wet-edge form, no averaging, no time-varying crest) */
  if (m->nfluxib) {
    std::fill(m->nib.begin(), m->nib.end(), 0);
    const double BARMIN = 0.04;
    const int *NODECODE = a->nodecode;
    auto NBV = [&](int I) { return a->nbv[I - 1] - 1; };        /* 1-based entry -> node */
    auto IBCONN = [&](int I) { return a->ibconn[I - 1] - 1; };
    int I = 0;
    for (int K = 0; K < a->nbou; ++K) {
      const int lb = a->lbcodei[I], NV = a->nvell[K];
      if (lb != 4 && lb != 24 && lb != 5 && lb != 25) {
        I = I + NV;
        continue;
      }
      for (int J = 1; J <= NV * 2; ++J) {
        I = I + 1;
        const int NNBB1 = NBV(I), NNBB2 = IBCONN(I);
        int NNBB1WN = 0, NNBB2WN = 0;
        if (J == 1 || J == NV + 1) {
          NNBB1WN = NNBB1WN + NODECODE[NBV(I + 1)];
          NNBB2WN = NNBB2WN + NODECODE[IBCONN(I + 1)];
        } else if (J == NV || J == NV * 2) {
          NNBB1WN = NNBB1WN + NODECODE[NBV(I - 1)];
          NNBB2WN = NNBB2WN + NODECODE[IBCONN(I - 1)];
        } else {
          NNBB1WN = NNBB1WN + NODECODE[NBV(I - 1)];
          NNBB1WN = NNBB1WN + NODECODE[NBV(I + 1)];
          NNBB2WN = NNBB2WN + NODECODE[IBCONN(I + 1)];
          NNBB2WN = NNBB2WN + NODECODE[IBCONN(I - 1)];
        }
        const double RBARWL1 = a->eta2[NNBB1] - a->barinht[I - 1];
        const double RBARWL2 = a->eta2[NNBB2] - a->barinht[I - 1];
        const double RBARWL1F = 2.0 * RBARWL1 / 3.0, RBARWL2F = 2.0 * RBARWL2 / 3.0;
        const double CFSB = a->barincfsb[I - 1], CFSP = a->barincfsp[I - 1];
        double FLUX = 0.0;
        if ((RBARWL1 < 0.0) && (RBARWL2 < 0.0)) {
          FLUX = 0.0;
        } else if (std::fabs(RBARWL1 - RBARWL2) < 0.01) {
          FLUX = 0.0;
        } else if ((RBARWL1 > RBARWL2) && (RBARWL1 > BARMIN)) {
          if (RBARWL2 > RBARWL1F) {
            if (NODECODE[NNBB1] == 0 || NNBB1WN == 0)
              FLUX = 0.0;
            else
              FLUX = -s->rampintflux * RBARWL2 * CFSB * std::sqrt(2.0 * G * (RBARWL1 - RBARWL2));
          } else {
            if (NODECODE[NNBB1] == 0 || NNBB1WN == 0)
              FLUX = 0.0;
            else
              FLUX = -s->rampintflux * CFSP * RBARWL1F * std::sqrt(RBARWL1F * G);
          }
        } else if ((RBARWL2 > RBARWL1) && (RBARWL2 > BARMIN)) {
          if (RBARWL1 > RBARWL2F) {
            if (NODECODE[NNBB2] == 0 || NNBB2WN == 0) {
              FLUX = 0.0;
            } else {
              FLUX = s->rampintflux * RBARWL1 * CFSB * std::sqrt(2.0 * G * (RBARWL2 - RBARWL1));
              m->nib[NNBB1] = 1;
            }
          } else {
            if (NODECODE[NNBB2] == 0 || NNBB2WN == 0) {
              FLUX = 0.0;
            } else {
              FLUX = s->rampintflux * CFSP * RBARWL2F * std::sqrt(RBARWL2F * G);
              m->nib[NNBB1] = 1;
            }
          }
        }
        m->qn2[I - 1] = FLUX;
      }
    }
  }
  /* discharge through cross-barrier pipes, timestep.F:1034-1044 and
   * COMPUTE_CROSS_BARRIER_PIPE_FLUX (weir_boundary.F90:2469-2579) */
  if (m->nfluxibp) {
    const double BARMIN = 0.04, PI = 3.141592653589793;
    const int *NODECODE = a->nodecode;
    for (int I = 0; I < a->nvel; ++I) {
      if (a->lbcodei[I] != 5 && a->lbcodei[I] != 25) continue;
      const int NNBB1 = a->nbv[I] - 1, NNBB2 = a->ibconn[I] - 1;
      const double PIPEHT = a->pipeht[I], PIPECOEF = a->pipecoef[I], PIPEDIAM = a->pipediam[I];
      const double RBARWL1 = a->eta2[NNBB1] - PIPEHT, RBARWL2 = a->eta2[NNBB2] - PIPEHT;
      double FLUX = 0.0;
      [&] {
        if ((RBARWL1 < 0.0) && (RBARWL2 < 0.0)) return;
        if (std::fabs(RBARWL1 - RBARWL2) < BARMIN) return;
        if ((RBARWL1 > RBARWL2) && (RBARWL1 > BARMIN)) {
          if (RBARWL2 <= 0.0) {
            if (NODECODE[NNBB1] == 0)
              FLUX = 0.0;
            else
              FLUX = -s->rampintflux * 0.25 * PI * (PIPEDIAM * PIPEDIAM) *
                     std::sqrt(2.0 * G * RBARWL1 / (1.0 + PIPECOEF));
          } else {
            if (NODECODE[NNBB1] == 0)
              FLUX = 0.0;
            else
              FLUX = -s->rampintflux * 0.25 * PI * (PIPEDIAM * PIPEDIAM) *
                     std::sqrt(2.0 * G * (RBARWL1 - RBARWL2) / PIPECOEF);
            return;
          }
        }
        if ((RBARWL2 > RBARWL1) && (RBARWL2 > BARMIN)) {
          if (RBARWL1 <= 0.0) {
            if (NODECODE[NNBB2] == 0) {
              FLUX = 0.0;
            } else {
              FLUX = s->rampintflux * 0.25 * PI * (PIPEDIAM * PIPEDIAM) *
                     std::sqrt(2.0 * G * RBARWL2 / (1.0 + PIPECOEF));
              m->nib[NNBB1] = 1;
            }
          } else {
            if (NODECODE[NNBB2] == 0) {
              FLUX = 0.0;
            } else {
              FLUX = s->rampintflux * 0.25 * PI * (PIPEDIAM * PIPEDIAM) *
                     std::sqrt(2.0 * G * (RBARWL2 - RBARWL1) / PIPECOEF);
              m->nib[NNBB1] = 1;
            }
          }
        }
      }();
      m->qn2[I] = m->qn2[I] + FLUX;
    }
  }
  /* zero normal velocity gradient entries, timestep.F:945-952 */
  if (m->nfluxgbc) {
    for (int J = 0; J < a->nvel; ++J) {
      if (a->lbcodei[J] != 40 && a->lbcodei[J] != 41) continue;
      const int NNBB = a->nbv[J] - 1;
      const double UN1 = a->uu1[NNBB] * a->csii[J] + a->vv1[NNBB] * a->siii[J];
      m->qn1[J] = a->h2[NNBB] * UN1;
    }
  }
}

/* GWCE_New, gwce.F:237-2111, IM=0 (KGQ lateral stress, NC advection),
 * ILump=0 consistent mass, Cartesian, no sponge/subgrid/flux BCs. */
int orc_model_gwce(orc_model *m, const orc_step_t *s, orc_stepout_t *out) {
  orc_arrays_t *a = m->a;
  const orc_params_t &p = m->p;
  const int np = a->np, ne = a->ne, mnei = a->mnei;
  const double DT = p.dt, G = p.g, A00 = p.a00, B00 = p.b00, C00 = p.c00;
  const int OnDiag = 2, OffDiag = 1; /* (1+ILump)*2, (1-ILump) */
  double *Coef = a->coef;
  auto COEF = [&](int i, int j) -> double & { return Coef[i + (size_t)np * j]; };
  int status = 0;

  if (m->ncchange > 0) {
    m->ncchange = 0;
    for (size_t k = 0; k < (size_t)np * mnei; ++k) Coef[k] = 0.0;
    par_for(ne, [&](int ie) {
      int n1 = NM(a, ie, 0), n2 = NM(a, ie, 1), n3 = NM(a, ie, 2);
      int NCEle = a->nodecode[n1] * a->nodecode[n2] * a->nodecode[n3] * a->noff[ie];
      double FDX1 = a->fdxe[3 * (size_t)ie], FDX2 = a->fdxe[3 * (size_t)ie + 1], FDX3 = a->fdxe[3 * (size_t)ie + 2];
      double FDY1 = a->fdye[3 * (size_t)ie], FDY2 = a->fdye[3 * (size_t)ie + 1], FDY3 = a->fdye[3 * (size_t)ie + 2];
      double AreaIE2 = a->areas[ie];
      double AreaIE = AreaIE2 * 0.5;
      double AreaIE4 = AreaIE2 * 2.0;
      double DPAvg = (a->dp[n1] + a->dp[n2] + a->dp[n3]) / 3.0 +
                     p.ifnlfa * 0 * (a->eta2[n1] + a->eta2[n2] + a->eta2[n3]) / 3.0;
      double GA00DPAvgOAreaIE4 = a->alphal[ie] * A00 * G * DPAvg * 1.0 / AreaIE4;
      double Tau0Avg = (a->tau0var[n1] + a->tau0var[n2] + a->tau0var[n3]) / 3.0;
      double MsFacLOnDiag = OnDiag * AreaIE * (1.0 / DT + Tau0Avg / 2.0) / DT / 12.0;
      double MsFacLOffDiag = OffDiag * AreaIE * (1.0 / DT + Tau0Avg / 2.0) / DT / 12.0;
      const int *cp = a->csr_position;
      int J12 = cp[ie + (size_t)ne * (0 + 3 * 0)] - 1;
      int J13 = cp[ie + (size_t)ne * (0 + 3 * 1)] - 1;
      int J21 = cp[ie + (size_t)ne * (1 + 3 * 0)] - 1;
      int J23 = cp[ie + (size_t)ne * (1 + 3 * 1)] - 1;
      int J31 = cp[ie + (size_t)ne * (2 + 3 * 0)] - 1;
      int J32 = cp[ie + (size_t)ne * (2 + 3 * 1)] - 1;
      double nc = (double)NCEle;
      orc_add(COEF(n1, 0), (MsFacLOnDiag + GA00DPAvgOAreaIE4 * (FDX1 * FDX1 + FDY1 * FDY1)) * nc);
      orc_add(COEF(n1, J12), (MsFacLOffDiag + GA00DPAvgOAreaIE4 * (FDX1 * FDX2 + FDY1 * FDY2)) * nc);
      orc_add(COEF(n1, J13), (MsFacLOffDiag + GA00DPAvgOAreaIE4 * (FDX1 * FDX3 + FDY1 * FDY3)) * nc);
      orc_add(COEF(n2, J21), (MsFacLOffDiag + GA00DPAvgOAreaIE4 * (FDX2 * FDX1 + FDY2 * FDY1)) * nc);
      orc_add(COEF(n2, 0), (MsFacLOnDiag + GA00DPAvgOAreaIE4 * (FDX2 * FDX2 + FDY2 * FDY2)) * nc);
      orc_add(COEF(n2, J23), (MsFacLOffDiag + GA00DPAvgOAreaIE4 * (FDX2 * FDX3 + FDY2 * FDY3)) * nc);
      orc_add(COEF(n3, J31), (MsFacLOffDiag + GA00DPAvgOAreaIE4 * (FDX3 * FDX1 + FDY3 * FDY1)) * nc);
      orc_add(COEF(n3, J32), (MsFacLOffDiag + GA00DPAvgOAreaIE4 * (FDX3 * FDX2 + FDY3 * FDY2)) * nc);
      orc_add(COEF(n3, 0), (MsFacLOnDiag + GA00DPAvgOAreaIE4 * (FDX3 * FDX3 + FDY3 * FDY3)) * nc);
    });
    /* gwce.F:646-650 */
    double EP = 0.0;
    for (int i = 0; i < np; ++i) EP = EP + COEF(i, 0) * COEF(i, 0);
    EP = std::sqrt(EP / np);
    m->ep = EP;
    /* gwce.F:654-673 */
    for (int I = 0; I < a->neta; ++I) {
      int b = a->nbd[I] - 1;
      COEF(b, 0) = EP;
      for (int J = 2; J <= a->nneigh[b]; ++J) COEF(b, J - 1) = 0.0;
    }
    for (size_t k = 0; k < (size_t)a->neta * (mnei - 1); ++k) a->obccoef[k] = 0.0;
    for (int I = 0; I < a->neta; ++I) {
      int b = a->nbd[I] - 1;
      for (int J = 2; J <= a->nneigh[b]; ++J) {
        int nb = a->neitab[b + (size_t)np * (J - 1)] - 1;
        for (int IJ = 2; IJ <= a->nneigh[nb]; ++IJ) {
          if (b == a->neitab[nb + (size_t)np * (IJ - 1)] - 1) {
            a->obccoef[I + (size_t)a->neta * (J - 2)] = COEF(nb, IJ - 1);
            COEF(nb, IJ - 1) = 0.0;
          }
        }
      }
    }
    /* gwce.F:678-707 */
    bool die = false;
    for (int i = 0; i < np; ++i) {
      if (COEF(i, 0) == 0.0) COEF(i, 0) = EP;
      if (COEF(i, 0) < 0.0) die = true;
    }
    if (die) status = 1;
  }

  /* RHS element loop, gwce.F:1000-1617 (NWS/NRS gate for PR1, WSX1) */
  const bool met = (p.nws != 0);
  par_for(ne, [&](int ie) {
    int n1 = NM(a, ie, 0), n2 = NM(a, ie, 1), n3 = NM(a, ie, 2);
    int NCEle = a->nodecode[n1] * a->nodecode[n2] * a->nodecode[n3] * a->noff[ie];
    double E0N1 = a->eta1[n1], E0N2 = a->eta1[n2], E0N3 = a->eta1[n3];
    double E1N1 = a->eta2[n1], E1N2 = a->eta2[n2], E1N3 = a->eta2[n3];
    double E1N1SQ = E1N1 * E1N1, E1N2SQ = E1N2 * E1N2, E1N3SQ = E1N3 * E1N3;
    double ESN1 = a->etas[n1], ESN2 = a->etas[n2], ESN3 = a->etas[n3];
    double U1N1 = a->uu1[n1], U1N2 = a->uu1[n2], U1N3 = a->uu1[n3];
    double V1N1 = a->vv1[n1], V1N2 = a->vv1[n2], V1N3 = a->vv1[n3];
    double QX1N1 = a->qx1[n1], QX1N2 = a->qx1[n2], QX1N3 = a->qx1[n3];
    double QY1N1 = a->qy1[n1], QY1N2 = a->qy1[n2], QY1N3 = a->qy1[n3];
    double H1N1 = a->h2[n1], H1N2 = a->h2[n2], H1N3 = a->h2[n3];
    double EVMN1 = a->evm[n1], EVMN2 = a->evm[n2], EVMN3 = a->evm[n3];
    double T0N1 = a->tau0var[n1], T0N2 = a->tau0var[n2], T0N3 = a->tau0var[n3];
    double Pr1N1 = 0.0, Pr1N2 = 0.0, Pr1N3 = 0.0;
    if (met) { Pr1N1 = a->pr1[n1]; Pr1N2 = a->pr1[n2]; Pr1N3 = a->pr1[n3]; }
    const double *tkm = a->tkm;
    double BSXN1 = tkm[3 * (size_t)n1] * QX1N1 + tkm[3 * (size_t)n1 + 2] * QY1N1;
    double BSYN1 = tkm[3 * (size_t)n1 + 2] * QX1N1 + tkm[3 * (size_t)n1 + 1] * QY1N1;
    double BSXN2 = tkm[3 * (size_t)n2] * QX1N2 + tkm[3 * (size_t)n2 + 2] * QY1N2;
    double BSYN2 = tkm[3 * (size_t)n2 + 2] * QX1N2 + tkm[3 * (size_t)n2 + 1] * QY1N2;
    double BSXN3 = tkm[3 * (size_t)n3] * QX1N3 + tkm[3 * (size_t)n3 + 2] * QY1N3;
    double BSYN3 = tkm[3 * (size_t)n3 + 2] * QX1N3 + tkm[3 * (size_t)n3 + 1] * QY1N3;
    double AreaIE2 = a->areas[ie];
    double AreaIE = AreaIE2 / 2.0;
    double AreaIE4 = 2.0 * AreaIE2;
    double FDX1 = a->fdxe[3 * (size_t)ie], FDX2 = a->fdxe[3 * (size_t)ie + 1], FDX3 = a->fdxe[3 * (size_t)ie + 2];
    double FDY1 = a->fdye[3 * (size_t)ie], FDY2 = a->fdye[3 * (size_t)ie + 1], FDY3 = a->fdye[3 * (size_t)ie + 2];
    double E0XGrad2A = E0N1 * FDX1 + E0N2 * FDX2 + E0N3 * FDX3;
    double E0YGrad2A = E0N1 * FDY1 + E0N2 * FDY2 + E0N3 * FDY3;
    double E1XGrad2A = E1N1 * FDX1 + E1N2 * FDX2 + E1N3 * FDX3;
    double E1YGrad2A = E1N1 * FDY1 + E1N2 * FDY2 + E1N3 * FDY3;
    double Tau0XGrad2A = T0N1 * FDX1 + T0N2 * FDX2 + T0N3 * FDX3;
    double Tau0YGrad2A = T0N1 * FDY1 + T0N2 * FDY2 + T0N3 * FDY3;
    /* Kolar-Gray lateral stress, gwce.F:1253-1263 */
    double EVMXGrad = (EVMN1 * FDX1 + EVMN2 * FDX2 + EVMN3 * FDX3) / AreaIE2;
    double EVMYGrad = (EVMN1 * FDY1 + EVMN2 * FDY2 + EVMN3 * FDY3) / AreaIE2;
    double EVMAvgODT = ((EVMN1 + EVMN2 + EVMN3) / 3.0) / DT;
    double MX = (EVMXGrad * (QX1N1 * FDX1 + QX1N2 * FDX2 + QX1N3 * FDX3) +
                 EVMYGrad * (QY1N1 * FDX1 + QY1N2 * FDX2 + QY1N3 * FDX3) -
                 EVMAvgODT * (ESN1 * FDX1 + ESN2 * FDX2 + ESN3 * FDX3)) / AreaIE2;
    double MY = (EVMXGrad * (QX1N1 * FDY1 + QX1N2 * FDY2 + QX1N3 * FDY3) +
                 EVMYGrad * (QY1N1 * FDY1 + QY1N2 * FDY2 + QY1N3 * FDY3) -
                 EVMAvgODT * (ESN1 * FDY1 + ESN2 * FDY2 + ESN3 * FDY3)) / AreaIE2;
    double CorifAvg = (a->corif[n1] + a->corif[n2] + a->corif[n3]) / 3.0;
    double Tau0Avg = (T0N1 + T0N2 + T0N3) / 3.0;
    double Tau0QXAvg = (T0N1 * QX1N1 + T0N2 * QX1N2 + T0N3 * QX1N3) / 3.0;
    double Tau0QYAvg = (T0N1 * QY1N1 + T0N2 * QY1N2 + T0N3 * QY1N3) / 3.0;
    double U1Avg = (U1N1 + U1N2 + U1N3) / 3.0;
    double V1Avg = (V1N1 + V1N2 + V1N3) / 3.0;
    double QX1Avg = (QX1N1 + QX1N2 + QX1N3) / 3.0;
    double QY1Avg = (QY1N1 + QY1N2 + QY1N3) / 3.0;
    double ESAvg = (ESN1 + ESN2 + ESN3) / 3.0;
    double DPAvg = (a->dp[n1] + a->dp[n2] + a->dp[n3]) / 3.0 + p.ifnlfa * 0 * (E1N1 + E1N2 + E1N3) / 3.0;
    double DPAvgS0 = (a->dp[n1] + a->dp[n2] + a->dp[n3]) / 3.0 + p.ifnlfa * 0 * (E0N1 + E0N2 + E0N3) / 3.0;
    double GDPAvgOAreaIE4 = a->alphal[ie] * G * DPAvg * 1.0 / AreaIE4;
    double GDPAvgOAreaIE4_S0 = a->alphal[ie] * G * DPAvgS0 * 1.0 / AreaIE4;
    double HAvg = (H1N1 + H1N2 + H1N3) / 3.0;
    double GHAvg = a->alphal[ie] * G * HAvg;
    double GHAvgOAreaIE2 = GHAvg / AreaIE2;
    double BSXAvg = (BSXN1 + BSXN2 + BSXN3) / 3.0;
    double BSYAvg = (BSYN1 + BSYN2 + BSYN3) / 3.0;
    double MXAvg = MX, MYAvg = MY;
    /* CorifAvg + IFNLCT*TANPHIAvg*U1Avg with TANPHI = 0 */
    double WSXAvg = 0.0, WSYAvg = 0.0;
    if (met) {
      WSXAvg = (1.0 * a->wsx1[n1] + 1.0 * a->wsx1[n2] + 1.0 * a->wsx1[n3]) / 3.0;
      WSYAvg = (1.0 * a->wsy1[n1] + 1.0 * a->wsy1[n2] + 1.0 * a->wsy1[n3]) / 3.0;
    }
    double MsFacR = AreaIE * (1.0 / DT - Tau0Avg / 2.0) / DT / 12.0;
    double GOAreaIE4 = a->alphal[ie] * G / AreaIE4;
    double Tau0SpaVar = (QX1Avg * Tau0XGrad2A + QY1Avg * Tau0YGrad2A) / 6.0;
    double A00pB00 = A00 + B00;
    /* gwce.F:1447-1468: TiP, Off, Disp, BC terms are 0 in this path */
    double JXAvg = CorifAvg * QY1Avg -
                   p.ifnlfa * GOAreaIE4 * (1 - 0) * (E1N1SQ * FDX1 + E1N2SQ * FDX2 + E1N3SQ * FDX3) -
                   GHAvgOAreaIE2 * ((Pr1N1 - 0.0 - 0.0) * FDX1 + (Pr1N2 - 0.0 - 0.0) * FDX2 + (Pr1N3 - 0.0 - 0.0) * FDX3) +
                   WSXAvg - BSXAvg + MXAvg - 0.0 - 0.0 + Tau0QXAvg;
    double JYAvg = -CorifAvg * QX1Avg -
                   p.ifnlfa * GOAreaIE4 * (1 - 0) * (E1N1SQ * FDY1 + E1N2SQ * FDY2 + E1N3SQ * FDY3) -
                   GHAvgOAreaIE2 * ((Pr1N1 - 0.0 - 0.0) * FDY1 + (Pr1N2 - 0.0 - 0.0) * FDY2 + (Pr1N3 - 0.0 - 0.0) * FDY3) +
                   WSYAvg - BSYAvg + MYAvg - 0.0 - 0.0 + Tau0QYAvg;
    /* NC advection, gwce.F:1471-1480 */
    JXAvg = JXAvg - p.ifnlct * (QX1Avg * (U1N1 * FDX1 + U1N2 * FDX2 + U1N3 * FDX3) +
                                QY1Avg * (U1N1 * FDY1 + U1N2 * FDY2 + U1N3 * FDY3)) / AreaIE2 +
            p.ifnlcat * U1Avg * ESAvg / DT;
    JYAvg = JYAvg - p.ifnlct * (QX1Avg * (V1N1 * FDX1 + V1N2 * FDX2 + V1N3 * FDX3) +
                                QY1Avg * (V1N1 * FDY1 + V1N2 * FDY2 + V1N3 * FDY3)) / AreaIE2 +
            p.ifnlcat * V1Avg * ESAvg / DT;
    /* gwce.F:1534-1610 */
    double T1 = (OnDiag * ESN1 + OffDiag * (ESN2 + ESN3)) * MsFacR -
                GDPAvgOAreaIE4_S0 * (C00 * (FDX1 * E0XGrad2A + FDY1 * E0YGrad2A)) -
                GDPAvgOAreaIE4 * (A00pB00 * (FDX1 * E1XGrad2A + FDY1 * E1YGrad2A)) +
                (JXAvg * FDX1 + JYAvg * FDY1) * 0.5 + Tau0SpaVar;
    double T2 = (OnDiag * ESN2 + OffDiag * (ESN1 + ESN3)) * MsFacR -
                GDPAvgOAreaIE4_S0 * (C00 * (FDX2 * E0XGrad2A + FDY2 * E0YGrad2A)) -
                GDPAvgOAreaIE4 * (A00pB00 * (FDX2 * E1XGrad2A + FDY2 * E1YGrad2A)) +
                (JXAvg * FDX2 + JYAvg * FDY2) * 0.5 + Tau0SpaVar;
    double T3 = (OnDiag * ESN3 + OffDiag * (ESN1 + ESN2)) * MsFacR -
                GDPAvgOAreaIE4_S0 * (C00 * (FDX3 * E0XGrad2A + FDY3 * E0YGrad2A)) -
                GDPAvgOAreaIE4 * (A00pB00 * (FDX3 * E1XGrad2A + FDY3 * E1YGrad2A)) +
                (JXAvg * FDX3 + JYAvg * FDY3) * 0.5 + Tau0SpaVar;
    double nc = (double)NCEle;
    orc_add(a->gwce_lv[n1], T1 * nc);
    orc_add(a->gwce_lv[n2], T2 * nc);
    orc_add(a->gwce_lv[n3], T3 * nc);
    (void)AreaIE;
  });

  /* gwce.F:1622-1631 */
  for (int i = 0; i < np; ++i) {
    a->eta1[i] = a->eta2[i];
    a->h1[i] = a->h2[i];
    a->eta2[i] = 0.0;
  }
  /* periodic elevation BC, gwce.F:1638-1651 */
  for (int J = 0; J < a->nbfr; ++J) {
    int NCYC = 0;
    if (a->per[J] != 0.0) NCYC = (int)(s->timeh / a->per[J]);
    double ARGJ = a->amig[J] * (s->timeh - NCYC * a->per[J]) + a->face[J];
    double RFF = a->ff[J] * s->rampelev;
    for (int I = 0; I < a->neta; ++I) {
      double ARG = ARGJ - a->efa[J + (size_t)a->nbfr * I];
      int b = a->nbd[I] - 1;
      a->eta2[b] = a->eta2[b] + a->emo[J + (size_t)a->nbfr * I] * RFF * std::cos(ARG);
    }
  }
  /* non-periodic elevation BC, gwce.F:1659-1674 */
  if (m->npebc) {
    if (s->timeloc > m->etime2) {
      m->etime1 = m->etime2;
      m->etime2 = m->etime1 + m->etiminc;
      if (m->e19_next >= m->e19_nrec) {   /* the reference's READ hits the end of fort.19 */
        m->series_err = 1;
      } else {
        const size_t r = (size_t)m->e19_next++ * a->neta;
        for (int J = 0; J < a->neta; ++J) {
          m->esbin1[J] = m->esbin2[J];
          m->esbin2[J] = m->e19[r + J];
        }
      }
    }
    const double ETRATIO = (s->timeloc - m->etime1) / m->etiminc;
    for (int I = 0; I < a->neta; ++I) {
      const int NBDI = a->nbd[I] - 1;
      a->eta2[NBDI] = a->eta2[NBDI] + s->rampelev * (m->esbin1[I] + ETRATIO * (m->esbin2[I] - m->esbin1[I]));
    }
  }
  /* boundary flux integral, gwce.F:1737-1834 (LBCODEI <= 29 types,
   * radiation 30 and river radiation 52, with the H1 saved above) */
  if (m->nfluxf || m->nfluxrbc || m->nfluxgbc || m->nfluxb || m->nfluxib) {
    const double DT2 = p.dt * 2.0;
    auto qforce = [&](int J, int NBDJ) {
      if (a->lbcodei[J] == 32) {   /* gwce.F:1792-1797 */
        const double CELERITY = std::sqrt(G * a->h1[NBDJ]);
        return (m->qn2[J] - m->qn0[J]) / DT2 -
               CELERITY * (2.0 * a->etas[NBDJ] - (m->en2[J] - m->en0[J])) / DT2 +
               a->tau0var[NBDJ] * (m->qn1[J] - CELERITY * (a->eta1[NBDJ] - m->en1[J]));
      }
      if (a->lbcodei[J] == 40 || a->lbcodei[J] == 41)   /* gwce.F:1804-1805 */
        return -(m->qn1[J] - m->qn0[J]) / DT - a->tau0var[NBDJ] * (m->qn1[J] + m->qn0[J]) / 2.0;
      if (a->lbcodei[J] == 30) {
        const double CELERITY = std::sqrt(G * a->h1[NBDJ]);
        return -CELERITY * a->etas[NBDJ] / DT - a->tau0var[NBDJ] * m->qn1[J];
      }
      double QforceJ = (m->qn2[J] - m->qn0[J]) / DT2 + a->tau0var[NBDJ] * m->qn1[J];
      if (a->lbcodei[J] == 52 && s->it > m->flux_settling_it) {
        const double Celerity = std::sqrt(G * a->h1[NBDJ]);
        QforceJ = QforceJ - Celerity * (a->etas[NBDJ] / DT +
                                        a->tau0var[NBDJ] * (a->eta1[NBDJ] - m->elevdisc[J]));
      }
      return QforceJ;
    };
    int NBDJ = a->nbv[0] - 1;
    double QFORCEJ = qforce(0, NBDJ);
    for (int J = 1; J < a->nvel; ++J) {
      const int NBDI = NBDJ;
      NBDJ = a->nbv[J] - 1;
      const double QFORCEI = QFORCEJ;
      QFORCEJ = qforce(J, NBDJ);
      const int NCI = a->nodecode[NBDI], NCJ = a->nodecode[NBDJ];
      const double B = NCI * NCJ * a->bndlen2o3[J - 1] / 4.0;
      a->gwce_lv[NBDI] = a->gwce_lv[NBDI] + B * (2.0 * QFORCEI + QFORCEJ);
      a->gwce_lv[NBDJ] = a->gwce_lv[NBDJ] + B * (2.0 * QFORCEJ + QFORCEI);
    }
  }
  /* elevation BC into the load vector, gwce.F:1846-1855 */
  for (int I = 0; I < a->neta; ++I) {
    int b = a->nbd[I] - 1;
    a->etas[b] = a->eta2[b] - a->eta1[b];
    a->gwce_lv[b] = a->etas[b] * a->nodecode[b] * m->ep;
    for (int J = 2; J <= a->nneigh[b]; ++J) {
      int nb = a->neitab[b + (size_t)np * (J - 1)] - 1;
      a->gwce_lv[nb] = a->gwce_lv[nb] - a->etas[b] * a->obccoef[I + (size_t)a->neta * (J - 2)];
    }
  }
  /* JCG, gwce.F:2002-2008 */
  m->iparm[0] = p.itmax;
  int ier = 0;
  int n = np, ndim = np, maxnz = mnei;
  jcg_impl(n, ndim, maxnz, const_cast<int *>(a->neitab), a->coef, a->gwce_lv, a->etas,
           m->iwksp.data(), m->nw, m->wksp.data(), m->iparm, m->rparm, ier);
  int numitr = m->iparm[0];
  for (int i = 0; i < np; ++i) a->eta2[i] = a->nodecode[i] * (a->etas[i] + 0.0) + a->eta1[i];
  if (out) {
    out->numitr = numitr;
    out->ier = ier;
    out->status = status;
    out->ep = m->ep;
    out->zeta = m->rparm[0];
    out->cme = m->rparm[1];
  }
  return status;
}

/* computeWettingAndDrying, wetdry.F:140-1470, non-subgrid, 2DDI, no weirs,
 * no barriers (NIBNODECODE = 0), NDDT = 0, default (non-SB_WETDRY) NOFF. */
int orc_model_wetdry(orc_model *m, const orc_step_t *s, orc_stepout_t *out) {
  (void)s;
  orc_arrays_t *a = m->a;
  const orc_params_t &p = m->p;
  const int np = a->np, ne = a->ne;
  if (p.nolifa != 2) {
    if (out) { out->ncchange = m->ncchange; out->n_w1_events = 0; }
    return 0;
  }
  const double H0 = p.h0, HABSMIN = 0.8 * H0, HOFF = 1.2 * H0, G = p.g;
  double *TK = a->tk, *TKM = a->tkm, *ETA2 = a->eta2;
  int *NODECODE = a->nodecode, *NNODECODE = a->nnodecode, *NOFF = a->noff;
  std::vector<double> &TK_TMP = m->tk_tmp;
  std::fill(TK_TMP.begin(), TK_TMP.end(), 0.0);
  const double TKNF = 1.0;
  std::vector<int> NOFFOLD(ne);
  for (int i = 0; i < ne; ++i) { NOFFOLD[i] = NOFF[i]; NOFF[i] = 1; }
  /* D1, wetdry.F:234-285 */
  for (int i = 0; i < np; ++i) {
    if (NODECODE[i] == 1) {
      double HTOT = a->dp[i] + ETA2[i];
      if (HTOT <= H0) {
        if (HTOT < HABSMIN) ETA2[i] = HABSMIN - a->dp[i];
        NNODECODE[i] = 0;
        NODECODE[i] = 0;
        m->ncchange = m->ncchange + 1;
      }
    }
  }
  /* W1, wetdry.F:332-809 */
  int nevents = 0;
  auto hyb = [&](double h1) {
    return p.ifhybf * std::pow(1.0 + std::pow(p.hbreak / h1, p.ftheta), p.fgamma / p.ftheta);
  };
  for (int ie = 0; ie < ne; ++ie) {
    int NM1 = NM(a, ie, 0), NM2 = NM(a, ie, 1), NM3 = NM(a, ie, 2);
    int NCTOT = NODECODE[NM1] + NODECODE[NM2] + NODECODE[NM3];
    if (NCTOT != 2) continue;
    double HTOTN1 = a->dp[NM1] + ETA2[NM1];
    double HTOTN2 = a->dp[NM2] + ETA2[NM2];
    double HTOTN3 = a->dp[NM3] + ETA2[NM3];
    int wa, wb, dry; /* the two wet nodes in reference order, and the dry one */
    double ha, hb;
    if (NODECODE[NM1] == 1 && NODECODE[NM2] == 1) {
      wa = NM1; wb = NM2; dry = NM3; ha = HTOTN1; hb = HTOTN2;
    } else if (NODECODE[NM2] == 1 && NODECODE[NM3] == 1) {
      wa = NM2; wb = NM3; dry = NM1; ha = HTOTN2; hb = HTOTN3;
    } else if (NODECODE[NM3] == 1 && NODECODE[NM1] == 1) {
      wa = NM3; wb = NM1; dry = NM2; ha = HTOTN3; hb = HTOTN1;
    } else {
      continue;
    }
    if (!((ha >= HOFF) && (hb >= HOFF))) continue;
    int NM123 = wa;
    if (ETA2[wb] > ETA2[wa]) NM123 = wb;
    double dy = a->y[dry] - a->y[NM123], dx = a->x[dry] - a->x[NM123];
    double DELDIST = std::sqrt(dy * dy + dx * dx);
    double DELETA = ETA2[NM123] - ETA2[dry];
    if (DELETA < 0.0) DELETA = 0.0;
    double H1 = ETA2[NM123] + a->dp[NM123];
    double TKWET = std::max(a->fric[NM123] * (p.iflinbf + (p.velmin / H1) * (p.ifnlbf + hyb(H1))), 0.0001);
    double VEL = G * (DELETA / DELDIST) / TKWET;
    if (VEL > p.velmin) {
      NNODECODE[dry] = 1;
      ++nevents;
      TK_TMP[NM123] = std::min(a->fric[NM123] * (p.iflinbf + (TKNF * VEL / H1) * (p.ifnlbf + hyb(H1))), 2.0 / p.dt);
      TK[NM123] = std::max(TK_TMP[NM123], TK[NM123]);
      TKM[3 * (size_t)NM123] = TK[NM123];
      TKM[3 * (size_t)NM123 + 1] = TK[NM123];
      /* the partner is the other wet node; the reference's branch on
       * NM123 == NM2 (resp. NM3) selects exactly this node */
      int P = (NM123 == wa) ? wb : wa;
      TK_TMP[P] = TK[NM123];
      TK[P] = std::max(TK_TMP[P], TK[P]);
      TKM[3 * (size_t)P] = TK[P];
      TKM[3 * (size_t)P + 1] = TK[P];
      if (TK_TMP[P] < TK[P]) {
        TK[NM123] = TK[P];
        TKM[3 * (size_t)NM123] = TK[NM123];
        TKM[3 * (size_t)NM123 + 1] = TK[NM123];
      }
    }
  }
  /* W2a, wetdry.F:813-816: the reference adds each element's NIBNODECODE
   * sum to its nodes' NIBCNT at the end of every W1 iteration; W1 does not
   * touch NIBNODECODE, so the same sums are taken in a loop of their own */
  std::vector<int> &NIBCNT = m->nibcnt;
  std::fill(NIBCNT.begin(), NIBCNT.end(), 0);
  if (m->nfluxib) {
    for (int ie = 0; ie < ne; ++ie) {
      int NM1 = NM(a, ie, 0), NM2 = NM(a, ie, 1), NM3 = NM(a, ie, 2);
      const int NBNCTOT = m->nib[NM1] + m->nib[NM2] + m->nib[NM3];
      NIBCNT[NM1] = NIBCNT[NM1] + NBNCTOT;
      NIBCNT[NM2] = NIBCNT[NM2] + NBNCTOT;
      NIBCNT[NM3] = NIBCNT[NM3] + NBNCTOT;
    }
    /* W2b, wetdry.F:1086-1090 */
    for (int i = 0; i < np; ++i)
      if (NIBCNT[i] > 0 && NNODECODE[i] == 0) NNODECODE[i] = 1;
  }
  /* DE1, wetdry.F:1110-1162 */
  for (int ie = 0; ie < ne; ++ie) {
    int NM1 = NM(a, ie, 0), NM2 = NM(a, ie, 1), NM3 = NM(a, ie, 2);
    if (NIBCNT[NM1] * NIBCNT[NM2] * NIBCNT[NM3] != 0) continue;   /* receiving barrier nodes */
    double ETAN1 = ETA2[NM1], ETAN2 = ETA2[NM2], ETAN3 = ETA2[NM3];
    double HTOTN1 = a->dp[NM1] + ETA2[NM1];
    double HTOTN2 = a->dp[NM2] + ETA2[NM2];
    double HTOTN3 = a->dp[NM3] + ETA2[NM3];
    if ((ETAN1 >= ETAN2) && (ETAN2 > ETAN3))
      if ((HTOTN1 < HOFF) || (HTOTN2 < HOFF)) NOFF[ie] = 0;
    if ((ETAN2 >= ETAN3) && (ETAN3 > ETAN1))
      if ((HTOTN2 < HOFF) || (HTOTN3 < HOFF)) NOFF[ie] = 0;
    if ((ETAN3 >= ETAN1) && (ETAN1 > ETAN2))
      if ((HTOTN3 < HOFF) || (HTOTN1 < HOFF)) NOFF[ie] = 0;
    if ((ETAN1 >= ETAN3) && (ETAN3 > ETAN2))
      if ((HTOTN1 < HOFF) || (HTOTN3 < HOFF)) NOFF[ie] = 0;
    if ((ETAN2 >= ETAN1) && (ETAN1 > ETAN3))
      if ((HTOTN2 < HOFF) || (HTOTN1 < HOFF)) NOFF[ie] = 0;
    if ((ETAN3 >= ETAN2) && (ETAN2 > ETAN1))
      if ((HTOTN3 < HOFF) || (HTOTN2 < HOFF)) NOFF[ie] = 0;
  }
  /* D2, wetdry.F:1361-1391 */
  for (int i = 0; i < np; ++i) { a->mju[i] = 0; a->totalarea[i] = 0.0; }
  for (int ie = 0; ie < ne; ++ie) {
    int NM1 = NM(a, ie, 0), NM2 = NM(a, ie, 1), NM3 = NM(a, ie, 2);
    int NCEle = NNODECODE[NM1] * NNODECODE[NM2] * NNODECODE[NM3] * NOFF[ie];
    double AreaEle = NCEle * a->areas[ie] / 2.0;
    a->mju[NM1] += NCEle; a->mju[NM2] += NCEle; a->mju[NM3] += NCEle;
    a->totalarea[NM1] = a->totalarea[NM1] + AreaEle;
    a->totalarea[NM2] = a->totalarea[NM2] + AreaEle;
    a->totalarea[NM3] = a->totalarea[NM3] + AreaEle;
  }
  for (int i = 0; i < np; ++i) {
    if (NNODECODE[i] == 1 && a->mju[i] == 0) NNODECODE[i] = 0;
    if (a->mju[i] == 0) a->mju[i] = 1;
  }
  /* wetdry.F:1413-1430 */
  for (int i = 0; i < np; ++i)
    if (NNODECODE[i] != NODECODE[i]) { NODECODE[i] = NNODECODE[i]; m->ncchange = m->ncchange + 1; }
  for (int ie = 0; ie < ne; ++ie)
    if (NOFF[ie] != NOFFOLD[ie]) m->ncchange = m->ncchange + 1;
  /* computeAlpha, wetdry.F:1561-1652 */
  for (int ie = 0; ie < ne; ++ie) a->alphal[ie] = 1.0;
  for (int ie = 0; ie < ne; ++ie) {
    int NM1 = NM(a, ie, 0), NM2 = NM(a, ie, 1), NM3 = NM(a, ie, 2);
    int NCEle = NODECODE[NM1] * NODECODE[NM2] * NODECODE[NM3] * NOFF[ie];
    if (NCEle != 1) continue;
    double HN1 = ETA2[NM1] + a->dp[NM1], HN2 = ETA2[NM2] + a->dp[NM2], HN3 = ETA2[NM3] + a->dp[NM3];
    if (!((HN1 <= 5.0e-1) || (HN2 <= 5.0e-1) || (HN3 <= 5.0e-1))) continue;
    double FDX1 = a->fdxe[3 * (size_t)ie], FDX2 = a->fdxe[3 * (size_t)ie + 1], FDX3 = a->fdxe[3 * (size_t)ie + 2];
    double FDY1 = a->fdye[3 * (size_t)ie], FDY2 = a->fdye[3 * (size_t)ie + 1], FDY3 = a->fdye[3 * (size_t)ie + 2];
    double ETAN1 = ETA2[NM1], ETAN2 = ETA2[NM2], ETAN3 = ETA2[NM3];
    double DPN1 = a->dp[NM1], DPN2 = a->dp[NM2], DPN3 = a->dp[NM3];
    double DPDXA = DPN1 * FDX1 + DPN2 * FDX2 + DPN3 * FDX3;
    double DPDYA = DPN1 * FDY1 + DPN2 * FDY2 + DPN3 * FDY3;
    double DETADXA = ETAN1 * FDX1 + ETAN2 * FDX2 + ETAN3 * FDX3;
    double DETADYA = ETAN1 * FDY1 + ETAN2 * FDY2 + ETAN3 * FDY3;
    double DPM = std::sqrt(DPDXA * DPDXA + DPDYA * DPDYA) / a->areas[ie];
    double al;
    if (DPM > 1.0e-5) {
      double DDTMP = DETADXA * (-DPDXA) + DETADYA * (-DPDYA);
      if (std::fabs(DDTMP) > 1.0e-12)
        al = p.slim * (std::sqrt(DPDXA * DPDXA + DPDYA * DPDYA) / ((1.0 / a->areas[ie]) * (DDTMP)));
      else
        al = 1.0;
    } else {
      double DETAM = std::sqrt(DETADXA * DETADXA + DETADYA * DETADYA) / a->areas[ie];
      if (std::fabs(DETAM) > 1.0e-12) al = p.slim / DETAM;
      else al = 1.0;
    }
    if (al <= 0.0) al = 1.0;
    if (al >= 1.0) al = 1.0;
    a->alphal[ie] = al;
  }
  if (out) { out->ncchange = m->ncchange; out->n_w1_events = nevents; }
  return 0;
}

/* gfortran's inline NORM2 for a rank-1 array (scaled sum of squares,
 * scale starting at 1); used by adcirc_norm2 (global.F:1502-1515). */
static double gf_norm2(const double *x, int n) {
  double scale = 1.0, result = 0.0;
  for (int i = 0; i < n; ++i) {
    if (x[i] != 0.0) {
      double absx = std::fabs(x[i]);
      if (scale < absx) {
        double val = scale / absx;
        result = 1.0 + result * val * val;
        scale = absx;
      } else {
        double val = absx / scale;
        result = result + val * val;
      }
    }
  }
  return scale * std::sqrt(result);
}

/* Mom_Eqs_New_NC, momentum.F:166-1208, IBPV lateral stress, corrected
 * area integration, land BCs LBCODEI 0-19, no sponge/condensed/VEW. */
int orc_model_momentum(orc_model *m, const orc_step_t *s) {
  (void)s;
  orc_arrays_t *a = m->a;
  const orc_params_t &p = m->p;
  const int np = a->np, ne = a->ne;
  const double DT = p.dt, G = p.g;
  const double THIRD = 1.0 / 3.0, GO2 = G / 2.0, DTO2 = DT / 2.0;
  const double Cfac1 = 1.0, Cfac2 = 1.0;
  const bool met = (p.nws != 0);
  par_for(ne, [&](int ie) {
    int n1 = NM(a, ie, 0), n2 = NM(a, ie, 1), n3 = NM(a, ie, 2);
    int NCEle = a->nodecode[n1] * a->nodecode[n2] * a->nodecode[n3] * a->noff[ie];
    double U1N1 = a->uu1[n1], U1N2 = a->uu1[n2], U1N3 = a->uu1[n3];
    double V1N1 = a->vv1[n1], V1N2 = a->vv1[n2], V1N3 = a->vv1[n3];
    double H1N1 = a->h1[n1], H1N2 = a->h1[n2], H1N3 = a->h1[n3];
    double AreaIE2 = a->areas[ie];
    double AreaIE = 0.5 * AreaIE2;
    double FDX1 = a->fdxe[3 * (size_t)ie], FDX2 = a->fdxe[3 * (size_t)ie + 1], FDX3 = a->fdxe[3 * (size_t)ie + 2];
    double FDY1 = a->fdye[3 * (size_t)ie], FDY2 = a->fdye[3 * (size_t)ie + 1], FDY3 = a->fdye[3 * (size_t)ie + 2];
    double U1Avg = THIRD * (U1N1 + U1N2 + U1N3);
    double V1Avg = THIRD * (V1N1 + V1N2 + V1N3);
    double DU1DXA = (U1N1 * FDX1 + U1N2 * FDX2 + U1N3 * FDX3) * 0.5;
    double DU1DYA = (U1N1 * FDY1 + U1N2 * FDY2 + U1N3 * FDY3) * 0.5;
    double DV1DXA = (V1N1 * FDX1 + V1N2 * FDX2 + V1N3 * FDX3) * 0.5;
    double DV1DYA = (V1N1 * FDY1 + V1N2 * FDY2 + V1N3 * FDY3) * 0.5;
    double EVMEle = THIRD * (a->evm[n1] + a->evm[n2] + a->evm[n3]);
    double al = a->alphal[ie];
    double BTP1N1 = al * a->eta1[n1], BTP2N1 = al * a->eta2[n1];
    double BTP1N2 = al * a->eta1[n2], BTP2N2 = al * a->eta2[n2];
    double BTP1N3 = al * a->eta1[n3], BTP2N3 = al * a->eta2[n3];
    if (met) {
      BTP1N1 = BTP1N1 + a->pr1[n1]; BTP2N1 = BTP2N1 + a->pr2[n1];
      BTP1N2 = BTP1N2 + a->pr1[n2]; BTP2N2 = BTP2N2 + a->pr2[n2];
      BTP1N3 = BTP1N3 + a->pr1[n3]; BTP2N3 = BTP2N3 + a->pr2[n3];
    }
    double DBTPDX1A = BTP1N1 * FDX1 + BTP1N2 * FDX2 + BTP1N3 * FDX3;
    double DBTPDX2A = BTP2N1 * FDX1 + BTP2N2 * FDX2 + BTP2N3 * FDX3;
    double DBTPDY1A = BTP1N1 * FDY1 + BTP1N2 * FDY2 + BTP1N3 * FDY3;
    double DBTPDY2A = BTP2N1 * FDY1 + BTP2N2 * FDY2 + BTP2N3 * FDY3;
    double DBTPDXA = 0.5 * (Cfac1 * DBTPDX1A + Cfac2 * DBTPDX2A);
    double DBTPDYA = 0.5 * (Cfac1 * DBTPDY1A + Cfac2 * DBTPDY2A);
    double U1AvgDU1DXA = U1Avg * DU1DXA, V1AvgDU1DYA = V1Avg * DU1DYA;
    double U1AvgDV1DXA = U1Avg * DV1DXA, V1AvgDV1DYA = V1Avg * DV1DYA;
    /* IBPV, momentum.F:534-554 */
    double DU1DX = DU1DXA / AreaIE, DU1DY = DU1DYA / AreaIE;
    double DV1DX = DV1DXA / AreaIE, DV1DY = DV1DYA / AreaIE;
    double EVMH1N1 = EVMEle * H1N1, EVMH1N2 = EVMEle * H1N2, EVMH1N3 = EVMEle * H1N3;
    double LSXXN1 = EVMH1N1 * DU1DX, LSXXN2 = EVMH1N2 * DU1DX, LSXXN3 = EVMH1N3 * DU1DX;
    double LSXYN1 = EVMH1N1 * DU1DY, LSXYN2 = EVMH1N2 * DU1DY, LSXYN3 = EVMH1N3 * DU1DY;
    double LSYXN1 = EVMH1N1 * DV1DX, LSYXN2 = EVMH1N2 * DV1DX, LSYXN3 = EVMH1N3 * DV1DX;
    double LSYYN1 = EVMH1N1 * DV1DY, LSYYN2 = EVMH1N2 * DV1DY, LSYYN3 = EVMH1N3 * DV1DY;
    double nc = (double)NCEle;
    /* momentum.F:584-666; DBCPD*A = 0, TANPHI = 0 */
    double A1 = nc * DT * (-p.ifnlct * (U1AvgDU1DXA + V1AvgDU1DYA) - GO2 * DBTPDXA - 0.0 -
                           (1.5 * (LSXXN1 * FDX1 + LSXYN1 * FDY1)) / H1N1);
    double A2 = nc * DT * (-p.ifnlct * (U1AvgDU1DXA + V1AvgDU1DYA) - GO2 * DBTPDXA - 0.0 -
                           (1.5 * (LSXXN2 * FDX2 + LSXYN2 * FDY2)) / H1N2);
    double A3 = nc * DT * (-p.ifnlct * (U1AvgDU1DXA + V1AvgDU1DYA) - GO2 * DBTPDXA - 0.0 -
                           (1.5 * (LSXXN3 * FDX3 + LSXYN3 * FDY3)) / H1N3);
    double B1 = nc * DT * (-p.ifnlct * (U1AvgDV1DXA + V1AvgDV1DYA) - GO2 * DBTPDYA - 0.0 -
                           (1.5 * (LSYXN1 * FDX1 + LSYYN1 * FDY1)) / H1N1);
    double B2 = nc * DT * (-p.ifnlct * (U1AvgDV1DXA + V1AvgDV1DYA) - GO2 * DBTPDYA - 0.0 -
                           (1.5 * (LSYXN2 * FDX2 + LSYYN2 * FDY2)) / H1N2);
    double B3 = nc * DT * (-p.ifnlct * (U1AvgDV1DXA + V1AvgDV1DYA) - GO2 * DBTPDYA - 0.0 -
                           (1.5 * (LSYXN3 * FDX3 + LSYYN3 * FDY3)) / H1N3);
    orc_add(a->mom_lv_x[n1], A1);
    orc_add(a->mom_lv_x[n2], A2);
    orc_add(a->mom_lv_x[n3], A3);
    orc_add(a->mom_lv_y[n1], B1);
    orc_add(a->mom_lv_y[n2], B2);
    orc_add(a->mom_lv_y[n3], B3);
  });
  /* nodal part, momentum.F:713-803 */
  std::vector<double> AUV(4 * (size_t)np);
  for (int i = 0; i < np; ++i) {
    int NCI = a->nodecode[i];
    if (a->totalarea[i] != 0.0) {
      a->mom_lv_x[i] = a->mom_lv_x[i] / a->totalarea[i];
      a->mom_lv_y[i] = a->mom_lv_y[i] / a->totalarea[i];
    }
    double WSX = 0.0, WSY = 0.0;
    if (met) {
      WSX = DTO2 * p.ifwind * (a->wsx1[i] / a->h1[i] + a->wsx2[i] / a->h2[i]);
      WSY = DTO2 * p.ifwind * (a->wsy1[i] / a->h1[i] + a->wsy2[i] / a->h2[i]);
    }
    double VCOEFXX = DTO2 * (a->tkm[3 * (size_t)i] + 0.0);
    double VCOEFYY = DTO2 * (a->tkm[3 * (size_t)i + 1] + 0.0);
    double CorifA = a->corif[i]; /* + IFNLCT*TANPHI*UU1 with TANPHI = 0 */
    double VCOEFXY = DTO2 * (a->tkm[3 * (size_t)i + 2] - CorifA);
    double VCOEFYX = DTO2 * (a->tkm[3 * (size_t)i + 2] + CorifA);
    a->mom_lv_x[i] = NCI * (a->mom_lv_x[i] + WSX + (1.0 - VCOEFXX) * a->uu1[i] - VCOEFXY * a->vv1[i]);
    a->mom_lv_y[i] = NCI * (a->mom_lv_y[i] + WSY + (1.0 - VCOEFYY) * a->vv1[i] - VCOEFYX * a->uu1[i]);
    AUV[4 * (size_t)i + 0] = 1.0 + VCOEFXX * NCI;
    AUV[4 * (size_t)i + 1] = 1.0 + VCOEFYY * NCI;
    AUV[4 * (size_t)i + 2] = VCOEFXY * NCI;
    AUV[4 * (size_t)i + 3] = VCOEFYX * NCI;
  }
  /* velocity BCs, momentum.F:810-933 (LBCODEI 0-9, 10-19 and 41) */
  const double sqrt2 = std::sqrt(2.0);
  for (int J = 0; J < a->nvelme; ++J) {
    int I = a->me2gw[J] - 1;
    int NBDI = a->nbv[I] - 1;
    int NCI = a->nodecode[NBDI];
    int lb = a->lbcodei[I];
    double *auv = &AUV[4 * (size_t)NBDI];
    double csi = a->csii[I], sii = a->siii[I];
    if (lb >= 0 && lb <= 9) {
      double VelNorm = -m->qn2[I] / a->h2[NBDI];
      if (std::fabs(gf_norm2(&a->tkm[3 * (size_t)NBDI], 3) - sqrt2 * a->tk[NBDI]) < DBL_EPSILON) {
        a->mom_lv_x[NBDI] = (sii * a->mom_lv_x[NBDI] - csi * a->mom_lv_y[NBDI] - VelNorm * auv[2]) * NCI;
        a->mom_lv_y[NBDI] = VelNorm * auv[0] * NCI;
        auv[2] = -csi * auv[0];
        auv[3] = -auv[2];
        auv[0] = sii * auv[0];
        auv[1] = auv[0];
      } else {
        a->mom_lv_x[NBDI] = (sii * a->mom_lv_x[NBDI] - csi * a->mom_lv_y[NBDI]) * NCI;
        a->mom_lv_y[NBDI] = VelNorm * NCI;
        auv[0] = auv[0] * sii - auv[3] * csi;
        auv[2] = auv[2] * sii - auv[1] * csi;
        auv[3] = csi;
        auv[1] = sii;
      }
    }
    if (lb >= 10 && lb <= 19) {
      double VelNorm = -m->qn2[I] / a->h2[NBDI];
      double VelTan = 0.0;
      a->mom_lv_x[NBDI] = VelTan * NCI;
      a->mom_lv_y[NBDI] = VelNorm * NCI;
      auv[0] = sii;
      auv[2] = -csi;
      auv[3] = csi;
      auv[1] = sii;
    }
    /* Galerkin zero normal velocity gradient, momentum.F:864-933 */
    if (lb == 41) {
      const int np_ = a->np;
      auto NeiTab = [&](int k) { return a->neitab[NBDI + (size_t)np_ * (k - 1)]; };
      auto NeiTabEle = [&](int k) { return a->neitabele[NBDI + (size_t)np_ * (k - 1)]; };
      auto FDXE = [&](int k, int e) { return a->fdxe[(k - 1) + 3 * (size_t)(e - 1)]; };
      auto FDYE = [&](int k, int e) { return a->fdye[(k - 1) + 3 * (size_t)(e - 1)]; };
      double ZNGRHS1 = 0.0, ZNGRHS2 = 0.0, ZNGLHS = 0.0;
      auto contribution = [&](int NM2, int NM3, int NEle) {
        if (NEle == 0) return;
        const int NCEle = NCI * a->nodecode[NM2 - 1] * a->nodecode[NM3 - 1] * a->noff[NEle - 1];
        if (NCEle == 0) return;
        const double sfdxfac = 1.0, sfdyfac = 1.0;   /* SFacEle = SFMXEle = SFMYEle = 1, IFSFM = 0 */
        const double FDX1 = FDXE(1, NEle) * sfdxfac, FDX2 = FDXE(2, NEle) * sfdxfac,
                     FDX3 = FDXE(3, NEle) * sfdxfac;
        const double FDY1 = FDYE(1, NEle) * sfdyfac, FDY2 = FDYE(2, NEle) * sfdyfac,
                     FDY3 = FDYE(3, NEle) * sfdyfac;
        ZNGRHS1 = ZNGRHS1 - (csi * FDX2 + sii * FDY2) * a->uu1[NM2 - 1] -
                  (csi * FDX3 + sii * FDY3) * a->uu1[NM3 - 1];
        ZNGRHS2 = ZNGRHS2 - (csi * FDX2 + sii * FDY2) * a->vv1[NM2 - 1] -
                  (csi * FDX3 + sii * FDY3) * a->vv1[NM3 - 1];
        ZNGLHS = ZNGLHS + csi * FDX1 + sii * FDY1;
      };
      int NM2 = NeiTab(2), NM3 = 0;
      const int NNFirst = NM2;
      const int nn = a->nneigh[NBDI];
      for (int N = 3; N <= nn; ++N) {
        NM3 = NM2;
        NM2 = NeiTab(N);
        contribution(NM2, NM3, NeiTabEle(N - 2));
      }
      NM3 = NM2;
      NM2 = NNFirst;
      contribution(NM2, NM3, NeiTabEle(nn - 1));
      if (NCI == 0) {
        a->mom_lv_x[NBDI] = 0.0;
        a->mom_lv_y[NBDI] = 0.0;
      } else {
        a->mom_lv_x[NBDI] = ZNGRHS1 / ZNGLHS;
        a->mom_lv_y[NBDI] = ZNGRHS2 / ZNGLHS;
      }
      auv[0] = 1.0;
      auv[1] = 1.0;
      auv[2] = 0.0;
      auv[3] = 0.0;
    }
  }
  /* 2x2 solve, momentum.F:1128-1138; fluxes :1179-1182 */
  for (int i = 0; i < np; ++i) {
    const double *auv = &AUV[4 * (size_t)i];
    double DDU = auv[0] * auv[1] - auv[2] * auv[3];
    a->uu2[i] = (a->mom_lv_x[i] * auv[1] - a->mom_lv_y[i] * auv[2]) / DDU;
    a->vv2[i] = (a->mom_lv_y[i] * auv[0] - a->mom_lv_x[i] * auv[3]) / DDU;
  }
  /* zero normal velocity gradient (IBTYPE 40), momentum.F:1157-1174 */
  if (m->nfluxgbc) {
    for (int J = 0; J < a->nvelme; ++J) {
      const int I = a->me2gw[J] - 1;
      if (a->lbcodei[I] != 40) continue;
      const int NBDI = a->nbv[I] - 1, E = a->nelezng[I] - 1;
      const int NM1 = a->nm[E] - 1, NM2 = a->nm[E + (size_t)a->ne] - 1,
                NM3 = a->nm[E + 2 * (size_t)a->ne] - 1;
      const int NCEle = a->nodecode[NM1] * a->nodecode[NM2] * a->nodecode[NM3] * a->noff[E];
      a->uu2[NBDI] = NCEle * (a->uu2[NM1] * a->zngif1[I] + a->uu2[NM2] * a->zngif2[I] +
                              a->uu2[NM3] * a->zngif3[I]);
      a->vv2[NBDI] = NCEle * (a->vv2[NM1] * a->zngif1[I] + a->vv2[NM2] * a->zngif2[I] +
                              a->vv2[NM3] * a->zngif3[I]);
    }
  }
  for (int i = 0; i < np; ++i) {
    a->qx2[i] = a->uu2[i] * a->h2[i];
    a->qy2[i] = a->vv2[i] * a->h2[i];
  }
  return 0;
}

int orc_model_set_vortex(orc_model *m, const orc_vortex_t *v) {
  if (!v || !v->fix || v->nfix < 2 || !(v->bladj > 0.0) || !(v->rho_air > 0.0)) return 1;
  for (int i = 1; i < v->nfix; ++i)
    if (!(v->fix[i].time > v->fix[i - 1].time)) return 1;
  /* NWS08INIT, nws08.F90:459-477 */
  int i0 = -1;
  for (int i = 1; i < v->nfix; ++i)
    if (std::ceil(v->start_time) >= v->fix[i - 1].time && std::floor(v->start_time) < v->fix[i].time) {
      i0 = i;
      break;
    }
  if (i0 < 0) return 1;
  m->vfix.assign(v->fix, v->fix + v->nfix);
  m->vpar = *v;
  m->vpar.fix = nullptr;
  m->vcounter = i0;
  m->vwtratio = 1.0;
  m->vortex_on = 1;
  return 0;
}

/* getMeteorologicalForcing for NWS = 8 on a Cartesian mesh: HollandGet
 * (nws08.F90:562-717; radial-velocity-weighted background wind, limited B,
 * no inflow angle, thetaLatDep false; Euclidean distance and atan2(dy,dx)
 * in mesh metres in place of the ICS = 2 haversine/DEG2RAD geometry) and
 * the NWS = 8 stress of wind.F:1172-1198 with capped Garratt drag
 * (wind.F:514-539). */
int orc_model_met(orc_model *m, const orc_step_t *s) {
  if (!m->vortex_on) return 0;
  orc_arrays_t *a = m->a;
  const orc_params_t &p = m->p;
  const orc_vortex_t &vp = m->vpar;
  const std::vector<orc_vortex_fix_t> &f = m->vfix;
  const double E = 2.718281828459045, ONE2TEN = 0.8928, PRB = 1013.0, RHOW = 1000.0;
  int err = 0;
  /* GetHollandStormData, nws08.F90:838-876 (position uses the previous
   * WTRATIO) */
  int i = m->vcounter;
  if (s->timeloc > f[i].time) {
    i = i + 1;
    if (i >= vp.nfix) { err = 1; i = vp.nfix - 1; }
  }
  const double lon = f[i - 1].x + m->vwtratio * (f[i].x - f[i - 1].x);
  const double lat = f[i - 1].y + m->vwtratio * (f[i].y - f[i - 1].y);
  /* a CALM line on either side (castType, nws08.F90:858-872; a negative
   * central pressure marks it): HollandGet returns zero wind and the
   * background pressure in metres of water (nws08.F90:588-601); WTRATIO is
   * not updated */
  if (f[i].cpress < 0.0 || f[i - 1].cpress < 0.0) {
    m->vcounter = i;
    const double prn2 = PRB * 100.0 / (RHOW * p.g);
    const double awr = vp.rho_air / RHOW;
    for (int n = 0; n < a->np; ++n) {
      const double wx = 0.0, wy = 0.0;
      const double mag = std::sqrt(wx * wx + wy * wy);
      const double drag = std::min(0.001 * (0.75 + 0.067 * mag), vp.drag_limit);
      a->wsx2[n] = s->rampmete * awr * drag * wx * mag;
      a->wsy2[n] = s->rampmete * awr * drag * wy * mag;
      a->pr2[n] = p.prbckgrnd_mh2o + s->rampmete * (prn2 - p.prbckgrnd_mh2o);
    }
    return err;
  }
  const double wt = (s->timeloc - f[i - 1].time) / (f[i].time - f[i - 1].time);
  m->vwtratio = wt;
  const double cpress = f[i - 1].cpress + wt * (f[i].cpress - f[i - 1].cpress);
  double spd = f[i - 1].vmax + wt * (f[i].vmax - f[i - 1].vmax);
  double rmw = f[i - 1].rmw + wt * (f[i].rmw - f[i - 1].rmw);
  const double tvx = f[i - 1].tvx + wt * (f[i].tvx - f[i - 1].tvx);
  const double tvy = f[i - 1].tvy + wt * (f[i].tvy - f[i - 1].tvy);
  m->vcounter = i;
  /* HollandGet, nws08.F90:616-639 */
  double dpdef = PRB * 100.0 - cpress;
  if (dpdef < 100.0) dpdef = 100.0;
  const double ts = std::sqrt(tvx * tvx + tvy * tvy);
  spd = spd - 1.0 * ts;
  spd = spd / vp.bladj;
  double B = vp.rho_air * E * (spd * spd) / dpdef;
  if (B < 1.0) B = 1.0;
  if (B > 2.5) B = 2.5;
  rmw = rmw * 1000.0;
  const double hemi = vp.hemisphere >= 0 ? 1.0 : -1.0;
  const double awr = vp.rho_air / RHOW;
  for (int n = 0; n < a->np; ++n) {
    /* nws08.F90:642-715 */
    const double dx = a->x[n] - lon, dy = a->y[n] - lat;
    const double theta = std::atan2(dy, dx);
    const double rad = std::sqrt(dx * dx + dy * dy);
    const double cf = a->corif[n];
    const double alpha = std::pow(rmw / rad, B);
    double press = cpress + dpdef * std::exp(-alpha);
    double vr = std::sqrt(alpha * std::exp(1.0 - alpha) * spd * (spd + 0.0) + 0.25 * (rad * rad) * (cf * cf)) -
                0.5 * rad * std::fabs(cf);
    vr = vr * vp.wind_mult;
    vr = vr * vp.bladj;
    double wx = (-hemi) * vr * std::sin(theta + hemi * 0.0);
    double wy = hemi * vr * std::cos(theta + hemi * 0.0);
    /* calcTranslationSpeed, nws08.F90:746-749 */
    wx = wx + (std::fabs(vr) / spd) * tvx;
    wy = wy + (std::fabs(vr) / spd) * tvy;
    if (vp.avg_minute == 1) {
      wx = wx * ONE2TEN;
      wy = wy * ONE2TEN;
    }
    press = std::max(0.85e5, std::min(1.1e5, press));
    wx = std::max(-200.0, std::min(200.0, wx));
    wy = std::max(-200.0, std::min(200.0, wy));
    const double prn2 = press / (RHOW * p.g);
    /* wind.F:1174-1193 */
    const double mag = std::sqrt(wx * wx + wy * wy);
    const double drag = std::min(0.001 * (0.75 + 0.067 * mag), vp.drag_limit);
    a->wsx2[n] = s->rampmete * awr * drag * wx * mag;
    a->wsy2[n] = s->rampmete * awr * drag * wy * mag;
    const double prdiff = s->rampmete * (prn2 - p.prbckgrnd_mh2o);
    a->pr2[n] = p.prbckgrnd_mh2o + prdiff;
  }
  return err;
}

int orc_model_step(orc_model *m, const orc_step_t *s, orc_stepout_t *out) {
  orc_stepout_t tmp;
  if (!out) out = &tmp;
  std::memset(out, 0, sizeof(*out));
  orc_model_shift_friction(m, s);
  if (orc_model_met(m, s)) { out->status = -1; return -1; }
  orc_model_flux(m, s);
  int st = orc_model_gwce(m, s, out);
  if (st != 0) return st;
  orc_model_wetdry(m, s, out);
  /* H2 update, timestep.F:1097-1099 */
  orc_arrays_t *a = m->a;
  for (int i = 0; i < a->np; ++i) a->h2[i] = a->dp[i] + m->p.ifnlfa * a->eta2[i];
  orc_model_momentum(m, s);
  out->ncchange = m->ncchange;
  if (m->series_err) { out->status = -1; return -1; }   /* past the end of fort.19/fort.20 */
  return 0;
}

/* Continue a run from another implementation's step-to-step state: the
 * module scalars NCChange, EP, RPARM(1:2), itjcg's SAVEd q1 and the NWS = 8
 * track position (bestTrackCounter, WTRATIO).  The arrays come in through
 * the bound orc_arrays_t. */
void orc_model_set_scalars(orc_model *m, int ncchange, double ep, double rparm1, double rparm2,
                           int q1, int vcounter, double vwtratio) {
  m->ncchange = ncchange;
  m->ep = ep;
  m->rparm[0] = rparm1;
  m->rparm[1] = rparm2;
  g_itp.q1 = (q1 != 0);
  if (m->vortex_on && vcounter >= 0) {
    m->vcounter = vcounter;
    m->vwtratio = vwtratio;
  }
}

void orc_coldstart(const orc_params_t *p, orc_arrays_t *a) {
  const int np = a->np, ne = a->ne;
  for (int i = 0; i < np; ++i) a->nnodecode[i] = 1;
  for (int i = 0; i < ne; ++i) a->noff[i] = 1;
  if (p->nolifa == 2) {
    for (int i = 0; i < np; ++i)
      if (a->dp[i] + a->eta2[i] <= p->h0) a->nnodecode[i] = 0;
    std::vector<int> mju(np, 0);
    for (int ie = 0; ie < ne; ++ie) {
      int n1 = NM(a, ie, 0), n2 = NM(a, ie, 1), n3 = NM(a, ie, 2);
      int nc = a->nnodecode[n1] * a->nnodecode[n2] * a->nnodecode[n3] * a->noff[ie];
      mju[n1] += nc; mju[n2] += nc; mju[n3] += nc;
    }
    for (int i = 0; i < np; ++i)
      if (a->nnodecode[i] == 1 && mju[i] == 0) a->nnodecode[i] = 0;
    for (int i = 0; i < np; ++i)
      if (a->nnodecode[i] == 0) a->eta2[i] = p->h0 - a->dp[i];
  }
  for (int i = 0; i < np; ++i) a->eta1[i] = a->eta2[i];
  /* totalAreaCalc, mesh.F:3360-3400 */
  for (int i = 0; i < np; ++i) { a->mju[i] = 0; a->totalarea[i] = 0.0; a->nodecode[i] = a->nnodecode[i]; }
  for (int ie = 0; ie < ne; ++ie) {
    int n1 = NM(a, ie, 0), n2 = NM(a, ie, 1), n3 = NM(a, ie, 2);
    int nc = a->nodecode[n1] * a->nodecode[n2] * a->nodecode[n3] * a->noff[ie];
    a->mju[n1] += nc; a->mju[n2] += nc; a->mju[n3] += nc;
    double ae = nc * a->areas[ie] / 2.0;
    a->totalarea[n1] = a->totalarea[n1] + ae;
    a->totalarea[n2] = a->totalarea[n2] + ae;
    a->totalarea[n3] = a->totalarea[n3] + ae;
  }
  for (int i = 0; i < np; ++i) if (a->mju[i] == 0) a->mju[i] = 1;
}

} /* extern "C" */
