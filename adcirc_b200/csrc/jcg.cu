// jcg.cu -- ITPACK 2D JCG (itpackv.F:63-604) as one persistent cooperative
// kernel on sm_100a.
//
// Design
//  * The scaled system (scal, itpackv.F:2281-2421) is built in-kernel from
//    the resident GWCE matrix, which also receives the reference's
//    scal/unscal rounding drift (itpackv.F:2447-2477) so a following solve
//    without a rebuild starts from the same bits.
//  * Each CG iteration is ONE grid-wide phase: a block updates u/d for its
//    rows (the 3-term recurrence, itpackv.F:593-596) and immediately forms
//    the next pseudo-residual SpMV (pjac, itpackv.F:1932-1967).  Neighbour
//    values of the new d are recomputed from the three previous buffers
//    (d rotates over 3 buffers, dtwd over 2) instead of waiting for their
//    owners, so the only grid barrier per iteration is the one the dot
//    products need.  The recomputation evaluates the same expression as
//    the owner, so every row sees identical bits.
//  * The dot products (sdot, itpackv.F:2828) are FP64 warp/block trees with
//    a fixed shape; the last block to reach the barrier reduces the block
//    partials in a fixed order and runs the scalar ITPACK steps
//    (pstop_nrms :809-890, parcon :1774-1851) on one thread.
//  * The adaptive eigenvalue estimate (chgcon :893-1027 with zbrent/determ)
//    only feeds the stopping test and depends only on the previous
//    iteration's scalars, so a dedicated extra block computes it while the
//    others run the SpMV, taking its latency off the critical path.
//  * Every barrier wait is bounded (clock64); on expiry the kernel records
//    a timeout and all blocks return.
#include "adc_internal.cuh"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>

namespace adc {

struct JcgArgs {
  int n, nslices, nrb, itmax;
  const int *sl_ptr, *sl_w, *col, *rlen;
  double *offd, *soff, *diag, *rhs;
  double *u, *u1, *d0, *d1, *d2, *t0, *t1, *w;
  double *part, *tri;
  Itp *itp;
  Bar *bar;
  Flags *flags;
  int eta_update;
  int do_peror;
  const int *nodecode;
  const double *eta1;
  double *eta2;
};

__device__ __forceinline__ double vld(const double *p) { return *(const volatile double *)p; }

// ---------------------------------------------------------------- barrier
// Returns true if this block was the last to arrive (only thread 0's view
// is meaningful; broadcast through shared memory by the caller).
__device__ bool bar_arrive(Bar *bar, unsigned nblocks, unsigned &gen_seen) {
  volatile unsigned *vgen = &bar->gen;
  gen_seen = *vgen;
  __threadfence();
  unsigned prev = atomicAdd(&bar->count, 1u);
  return prev == nblocks - 1;
}

__device__ void bar_release(Bar *bar) {
  bar->count = 0;
  __threadfence();
  atomicAdd(&bar->gen, 1u);
}

__device__ bool bar_wait(Bar *bar, unsigned gen_seen, Flags *flags) {
  volatile unsigned *vgen = &bar->gen;
  long long t0 = clock64();
  while (*vgen == gen_seen) {
    if (*(volatile int *)&flags->timeout) return false;
    if (clock64() - t0 > kSpinCycles) {
      atomicExch(&flags->timeout, 1);
      return false;
    }
    __nanosleep(64);
  }
  __threadfence();
  return true;
}

// Plain grid barrier.  Returns false on timeout.
__device__ bool grid_sync(const JcgArgs &a) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned g;
    bool last = bar_arrive(a.bar, gridDim.x, g);
    if (last) {
      bar_release(a.bar);
      ok = 1;
    } else {
      ok = bar_wait(a.bar, g, a.flags) ? 1 : 0;
    }
  }
  __syncthreads();
  return ok != 0;
}

// ---------------------------------------------------------------- scalars
__device__ double determ_d(int ldt, int n, const double *tri, double *wk1, double *wk2,
                           double xlmda) {
  for (int i = 1; i <= n; ++i) wk1[i - 1] = tri[i - 1] - xlmda;
  wk2[n - 1] = wk1[n - 1];
  wk2[n - 2] = wk1[n - 2] * wk2[n - 1] + tri[ldt + n - 1];
  if (n != 2)
    for (int l = n - 2; l >= 1; --l) wk2[l - 1] = wk1[l - 1] * wk2[l] + tri[ldt + l] * wk2[l + 1];
  return wk2[0];
}

// zbrent (itpackv.F:2521-2781): Brent root of the characteristic
// polynomial of the CG tridiagonal on [a, b].
__device__ void zbrent_d(int n, double *tri, int itmax, double eps, double t, double &a,
                         double &b, int &maxfn, int &ier) {
  double c = 0, d = 0, e = 0, p, q, r, s, fa, fb, fc, tol, rm, rone, temp;
  ier = 0;
  double *wk1 = tri + 2 * itmax, *wk2 = tri + 3 * itmax;
  int ic = 2;
  fa = determ_d(itmax, n, tri, wk1, wk2, a);
  fb = determ_d(itmax, n, tri, wk1, wk2, b);
  s = b;
  if ((fa > 0.0 && fb > 0.0) || (fa < 0.0 && fb < 0.0)) {
    ier = 502;
    maxfn = ic;
    return;
  }
  bool reset = true;
  for (;;) {
    if (reset) {
      c = a;
      fc = fa;
      d = b - c;
      e = d;
    }
    reset = false;
    if (!(fabs(fc) >= fabs(fb))) {
      a = b; b = c; c = a;
      fa = fb; fb = fc; fc = fa;
    }
    tol = t * fmax(fabs(b), 0.1);
    rm = (c - b) * 0.5;
    if (fabs(fb) <= eps || fabs(c - b) <= tol) {
      a = c;
      maxfn = ic;
      return;
    }
    if (ic >= maxfn) {
      ier = 501;
      a = c;
      maxfn = ic;
      return;
    }
    bool bisect = false;
    if (fabs(e) < tol || fabs(fa) <= fabs(fb)) {
      bisect = true;
    } else {
      s = fb / fa;
      if (a == c) {
        p = (c - b) * s;
        q = 1.0 - s;
      } else {
        q = fa / fc;
        r = fb / fc;
        rone = r - 1.0;
        p = s * ((c - b) * q * (q - r) - (b - a) * rone);
        q = (q - 1.0) * rone * (s - 1.0);
      }
      if (p > 0.0) q = -q;
      if (p < 0.0) p = -p;
      s = e;
      e = d;
      if (p + p >= 3.0 * rm * q || p + p >= fabs(s * q)) {
        bisect = true;
      } else {
        d = p / q;
      }
    }
    if (bisect) {
      e = rm;
      d = e;
    }
    a = b;
    fa = fb;
    temp = d;
    if (fabs(temp) <= 0.5 * tol) temp = copysign(0.5 * tol, rm);
    b = b + temp;
    s = b;
    fb = determ_d(itmax, n, tri, wk1, wk2, s);
    ic = ic + 1;
    if (fb == 0.0 || fc == 0.0) continue;
    if ((fb > 0.0 && fc < 0.0) || (fb < 0.0 && fc > 0.0)) continue;
    reset = true;
  }
}

// int(-log10(zeta)) as a glibc-linked Fortran build evaluates it: the
// logarithm rounded to the nearest double, then truncated.  Values within
// 1e-12 of an integer are taken as that integer (the correctly rounded
// logarithm of a double nearest a power of ten is that integer).
__device__ int nsig_of(double zeta) {
  double L = -log10(fabs(zeta));
  double k = rint(L);
  int itmp = (fabs(L - k) <= 1e-12 * fmax(1.0, fabs(k))) ? (int)k : (int)L;
  return itmp > 4 ? itmp : 4;
}

__device__ double pow10_neg(int nsig) {
  double p = 1.0;
  for (int i = 0; i < nsig; ++i) p *= 10.0;   // exact up to 1e22
  return 1.0 / p;
}

// chgcon, jacobi case (itpackv.F:893-1027), for iteration `in`.
__device__ void chgcon_d(volatile Itp *it, double *tri, int in) {
  const int ldt = it->itmax;
  double start = it->cme, end1 = 0.0;
  int ip = in;
  if (ip == 0) {
    it->cmold = 0.0;
    it->cme = 0.0;
    return;
  }
  if (ip == 1) {
    end1 = 1.0 - 1.0 / it->gamma;
    tri[0] = end1;
    tri[ldt] = 0.0;
    it->cme = end1;
    return;
  }
  if (fabs(start - it->cmold) <= it->zeta * start) {
    it->adapt = 0;
    return;
  }
  it->cmold = start;
  tri[ip - 1] = 1.0 - 1.0 / it->gamma;
  tri[ldt + ip - 1] = (1.0 - it->rho) / (it->rho * it->rhoold * it->gamma * it->gamold);
  int ier = 0;
  if (it->isym != 0) {
    ier = 903;
  } else {
    int nsig = nsig_of(it->zeta);
    int maxfn = it->itmax > 50 ? it->itmax : 50;
    double a = start, b = 1.0;
    zbrent_d(ip, tri, it->itmax, 0.0, pow10_neg(nsig), a, b, maxfn, ier);
    end1 = b;
  }
  it->chg_ier = ier;
  if (ier != 0) {
    it->adapt = 0;
    return;
  }
  it->cme = end1;
}

// pstop_nrms (itpackv.F:809-890, iflag = 1) for iteration `in`.
__device__ void pstop_d(volatile Itp *it, int in, double unrm, double dnrm) {
  double con = it->cme, uold, tr, tl;
  it->halt = 0;
  if (in < 1) {
    it->q1 = 0;
    it->udnm = 1.0;
    it->stptst = 1000.0;
  }
  if (!it->q1 && !((in > 5) && (in % 5 != 0))) {
    uold = it->udnm;
    it->udnm = unrm;
    if (it->udnm == 0.0) it->udnm = 1.0;
    if ((in > 5) && (fabs(it->udnm - uold) <= it->udnm * it->zeta)) it->q1 = 1;
  }
  tr = sqrt(it->udnm);
  tl = 1.0;
  if (con != 1.0) {
    tl = sqrt(dnrm);
    tr = tr * (1.0 - con);
  }
  it->stptst = tl / tr;
  if (tl >= tr * it->zeta) return;
  it->halt = 1;
}

// parcon (itpackv.F:1774-1851) for iteration `in`.
__device__ void parcon_d(volatile Itp *it, int in, double dtnrm) {
  double rhoold = it->rho;
  double gamold = it->gamma;
  it->gamma = 1.0 / (1.0 - dtnrm / it->delnnm);
  it->rho = 1.0;
  if (in != 0) it->rho = 1.0 / (1.0 - it->gamma * it->delnnm / (gamold * it->delsnm * rhoold));
  it->delsnm = it->delnnm;
  it->gamold = gamold;
  it->rhoold = rhoold;
  it->c1 = it->rho * it->gamma;
  it->c2 = it->rho;
  it->c3 = 1.0 - it->rho;
  it->c4 = it->rho * (1.0 - it->gamma);
}

// ------------------------------------------------------------ reductions
// Block-level fixed-tree sum of up to 3 values; result valid in thread 0.
__device__ void block_sum3(double &a, double &b, double &c) {
  __shared__ double sh[3][32];
  a = warp_sum(a);
  b = warp_sum(b);
  c = warp_sum(c);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) { sh[0][wid] = a; sh[1][wid] = b; sh[2][wid] = c; }
  __syncthreads();
  if (wid == 0) {
    a = lane < nw ? sh[0][lane] : 0.0;
    b = lane < nw ? sh[1][lane] : 0.0;
    c = lane < nw ? sh[2][lane] : 0.0;
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
  }
  __syncthreads();
}

// Reducing barrier: every block posts 3 partials; the last block to arrive
// sums them in a fixed order, runs `scalar(sum0, sum1, sum2)` on thread 0
// and releases the others.  Returns false on timeout.
template <class F>
__device__ bool reduce_sync(const JcgArgs &a, double p0, double p1, double p2, F scalar) {
  __shared__ int last_sh, ok_sh;
  block_sum3(p0, p1, p2);
  if (threadIdx.x == 0) {
    a.part[4 * blockIdx.x + 0] = p0;
    a.part[4 * blockIdx.x + 1] = p1;
    a.part[4 * blockIdx.x + 2] = p2;
  }
  __syncthreads();
  unsigned g = 0;
  if (threadIdx.x == 0) {
    last_sh = bar_arrive(a.bar, gridDim.x, g) ? 1 : 0;
    ok_sh = 1;
  }
  __syncthreads();
  if (last_sh) {
    __threadfence();
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
      s0 += vld(&a.part[4 * b + 0]);
      s1 += vld(&a.part[4 * b + 1]);
      s2 += vld(&a.part[4 * b + 2]);
    }
    block_sum3(s0, s1, s2);
    if (threadIdx.x == 0) {
      scalar(s0, s1, s2);
      __threadfence();
      bar_release(a.bar);
    }
  } else if (threadIdx.x == 0) {
    ok_sh = bar_wait(a.bar, g, a.flags) ? 1 : 0;
  }
  __syncthreads();
  return ok_sh != 0;
}

// ------------------------------------------------------------ the kernel
__global__ void __launch_bounds__(kThreads) jcg_kernel(JcgArgs a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const bool scalar_block = (blockIdx.x == (unsigned)a.nrb);
  const int s0 = scalar_block ? 0 : (int)((long long)a.nslices * blockIdx.x / a.nrb);
  const int s1 = scalar_block ? 0 : (int)((long long)a.nslices * (blockIdx.x + 1) / a.nrb);
  volatile Itp *vit = a.itp;
  volatile Itp *it = a.itp;
  const int n = a.n;

  // P0: scal part 1 -- u' = u*sqrt(d), w = 1/sqrt(d), rhs' = rhs*w.
  for (int s = s0 + warp; s < s1; s += nwarps) {
    int i = s * kSlice + lane;
    if (i < n) {
      double work = sqrt(a.diag[i]);
      a.u[i] = a.u[i] * work;
      double wv = 1.0 / work;
      a.w[i] = wv;
      a.rhs[i] = a.rhs[i] * wv;
      a.u1[i] = 0.0;
      a.d2[i] = 0.0;
    }
  }
  if (!grid_sync(a)) return;

  // P1: scaled off-diagonals, the reference's unscal drift of the resident
  // matrix, and the initial pseudo-residual d0 = pjac(u') + rhs' - u'.
  for (int s = s0 + warp; s < s1; s += nwarps) {
    int i = s * kSlice + lane;
    if (i < n) {
      int len = a.rlen[i];
      int base = a.sl_ptr[s] + lane;
      double wi = a.w[i];
      double winv_i = 1.0 / wi;
      double acc = a.rhs[i];
      for (int k = 0; k < len; ++k) {
        int idx = base + k * kSlice;
        int j = a.col[idx];
        double wj = a.w[j];
        double sv = a.offd[idx] * wi * wj;
        a.soff[idx] = sv;
        a.offd[idx] = sv * winv_i * (1.0 / wj);
        acc = acc - sv * a.u[j];
      }
      a.d0[i] = acc - a.u[i];
      a.diag[i] = winv_i * winv_i;
    }
  }
  if (!grid_sync(a)) return;

  // P2: dtwd0 = -A' d0 and the iteration-0 norms; the scalar block runs
  // chgcon for in = 0 (ip = 0: cme = 0).
  {
    double pd = 0.0, pt = 0.0, pu = 0.0;
    const int need_u = vit->need_unorm;
    for (int s = s0 + warp; s < s1; s += nwarps) {
      int i = s * kSlice + lane;
      if (i < n) {
        int len = a.rlen[i];
        int base = a.sl_ptr[s] + lane;
        double acc = 0.0;
        for (int k = 0; k < len; ++k) {
          int idx = base + k * kSlice;
          acc = acc - a.soff[idx] * a.d0[a.col[idx]];
        }
        a.t0[i] = acc;
        double di = a.d0[i];
        pd += di * di;
        pt += di * acc;
        if (need_u) { double ui = a.u[i]; pu += ui * ui; }
      }
    }
    if (scalar_block && threadIdx.x == 0 && it->adapt) chgcon_d(it, a.tri, 0);
    bool ok = reduce_sync(a, pd, pt, pu, [&](double sd, double st, double su) {
      it->delnnm = sd;
      double unorm = need_u ? su : 1.0;
      pstop_d(it, 0, unorm, sd);
      it->in = 0;
      if (!it->halt) {
        if (it->itmax == 0) {
          it->halt = 2;   // not converged at in = itmax
        } else {
          parcon_d(it, 0, st);
          it->need_unorm = !(it->q1 || ((1 > 5) && (1 % 5 != 0)));
        }
      }
    });
    if (!ok) return;
  }

  // Iteration phases.
  double *D[3] = {a.d0, a.d1, a.d2};
  double *T[2] = {a.t0, a.t1};
  double *U[2] = {a.u, a.u1};
  for (int in = 0; in < a.itmax; ++in) {
    if (vit->halt) break;
    const double c1 = vit->c1, c2 = vit->c2, c3 = vit->c3, c4 = vit->c4;
    const int need_u = vit->need_unorm;
    const double *dc = D[in % 3], *dp = D[(in + 2) % 3], *tc = T[in % 2];
    double *dn = D[(in + 1) % 3], *tn = T[(in + 1) % 2];
    const double *uc = U[in % 2];
    double *un = U[(in + 1) % 2];
    double pd = 0.0, pt = 0.0, pu = 0.0;
    for (int s = s0 + warp; s < s1; s += nwarps) {
      int i = s * kSlice + lane;
      if (i < n) {
        double unew = c1 * dc[i] + c2 * uc[i] + c3 * un[i];
        double dnew = c1 * tc[i] + c4 * dc[i] + c3 * dp[i];
        int len = a.rlen[i];
        int base = a.sl_ptr[s] + lane;
        double acc = 0.0;
        for (int k = 0; k < len; ++k) {
          int idx = base + k * kSlice;
          int j = a.col[idx];
          double dj = c1 * tc[j] + c4 * dc[j] + c3 * dp[j];
          acc = acc - a.soff[idx] * dj;
        }
        un[i] = unew;
        dn[i] = dnew;
        tn[i] = acc;
        pd += dnew * dnew;
        pt += dnew * acc;
        if (need_u) pu += unew * unew;
      }
    }
    const int m = in + 1;
    if (scalar_block && threadIdx.x == 0 && it->adapt) chgcon_d(it, a.tri, m);
    bool ok = reduce_sync(a, pd, pt, pu, [&](double sd, double st, double su) {
      it->delnnm = sd;
      double unorm = need_u ? su : 1.0;
      pstop_d(it, m, unorm, sd);
      it->in = m;
      if (!it->halt) {
        if (m >= it->itmax) {
          it->halt = 2;
        } else {
          parcon_d(it, m, st);
          int mm = m + 1;
          it->need_unorm = !(it->q1 || ((mm > 5) && (mm % 5 != 0)));
        }
      }
    });
    if (!ok) return;
  }

  const int fin = vit->in;
  const double *usol = U[fin % 2];

  // Optional peror (itpackv.F:607-720): the norms behind digit1/digit2.
  // pmult (itpackv.F:1970-2005) forms c = u - sum_j coef(:,j) u(jcoef).
  if (a.do_peror) {
    double pb = 0.0, pr = 0.0;
    for (int s = s0 + warp; s < s1; s += nwarps) {
      int i = s * kSlice + lane;
      if (i < n) {
        double wv = a.w[i];
        double wk = a.rhs[i] / wv;
        pb += wk * wk;
        int len = a.rlen[i];
        int base = a.sl_ptr[s] + lane;
        double cc = usol[i];
        for (int k = 0; k < len; ++k) {
          int idx = base + k * kSlice;
          cc = cc - a.soff[idx] * usol[a.col[idx]];
        }
        double wk2 = (a.rhs[i] - cc) / wv;
        pr += wk2 * wk2;
      }
    }
    bool ok = reduce_sync(a, pb, pr, 0.0, [&](double sb, double sr, double) {
      it->dtnrm = sb;
      it->unorm = sr;
    });
    if (!ok) return;
  }

  // Epilogue: unscal (itpackv.F:2447-2477) and the GWCE eta update
  // (gwce.F:2006-2008).
  for (int s = s0 + warp; s < s1; s += nwarps) {
    int i = s * kSlice + lane;
    if (i < n) {
      double wv = a.w[i];
      double uf = usol[i] * wv;
      a.u[i] = uf;
      a.rhs[i] = a.rhs[i] * (1.0 / wv);
      if (a.eta_update) a.eta2[i] = a.nodecode[i] * (uf + 0.0) + a.eta1[i];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int h = vit->halt;
    a.flags->numitr = fin;
    a.flags->ier = (h == 2) ? 13 : 0;
    if (h == 2) it->rparm1 = vit->stptst;   // itpackv.F:394
    a.flags->zeta = vit->rparm1;
    a.flags->cme = vit->cme;
  }
}

// Per-solve ITPACK initialisation (echall, itpackv.F:1212-1255, plus the
// zeta floor of jcg :223-232); q1 and rparm1 persist across solves.
__global__ void jcg_init_kernel(Itp *it, Bar *bar, int itmax) {
  bar->count = 0;
  it->zeta = it->rparm1;
  // cme keeps rparm(2) of the previous solve; chgcon(0) resets it to 0
  it->sme = -1.0;
  it->itmax = itmax;
  it->adapt = 1;
  it->isym = 0;
  it->in = 0;
  it->halt = 0;
  it->delnnm = it->delsnm = it->gamma = it->rho = it->stptst = it->udnm = 0.0;
  double temp = 512.0 * DBL_EPSILON;
  if (it->zeta < temp) it->zeta = temp;
  it->need_unorm = !(it->q1 || 0);
}

}  // namespace adc

using namespace adc;

namespace adc {

int jcg_setup_grid(adc_ctx *c) {
  int dev = 0, nsm = 0, per_sm = 0;
  ADC_CUDA(cudaGetDevice(&dev));
  ADC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  ADC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jcg_kernel, kThreads, 0));
  if (per_sm < 1) { set_error("jcg kernel cannot be resident"); return ADC_ERR_CUDA; }
  long long maxb = (long long)per_sm * nsm;
  int nrb = (int)std::min<long long>(maxb - 1, c->nslices);
  // keep at least ~8 slices per block so barrier cost stays amortised
  nrb = std::max(1, std::min(nrb, std::max(1, c->nslices / 8)));
  if (nrb > maxb - 1) nrb = (int)(maxb - 1);
  c->jcg_rows_blocks = nrb;
  c->jcg_grid = nrb + 1;
  return ADC_OK;
}

int launch_jcg_impl(adc_ctx *c, int eta_update, int do_peror, int run_init) {
  JcgArgs a;
  a.do_peror = do_peror;
  a.n = c->np;
  a.nslices = c->nslices;
  a.nrb = c->jcg_rows_blocks;
  a.itmax = c->itmax;
  a.sl_ptr = c->sl_ptr;
  a.sl_w = c->sl_w;
  a.col = c->col;
  a.rlen = c->rlen;
  a.offd = c->offd;
  a.soff = c->soff;
  a.diag = c->diag;
  a.rhs = c->gwce_lv;
  a.u = c->etas;
  a.u1 = c->ju1;
  a.d0 = c->jd[0];
  a.d1 = c->jd[1];
  a.d2 = c->jd[2];
  a.t0 = c->jdt[0];
  a.t1 = c->jdt[1];
  a.w = c->jw;
  a.part = c->jpart;
  a.tri = c->jtri;
  a.itp = c->itp;
  a.bar = c->bar;
  a.flags = c->flags;
  a.eta_update = eta_update;
  a.nodecode = c->nodecode;
  a.eta1 = c->eta1;
  a.eta2 = c->eta2;
  if (run_init) {
    jcg_init_kernel<<<1, 1, 0, c->stream>>>(c->itp, c->bar, c->itmax);
    c->launches++;
  }
  void *args[] = {&a};
  ADC_CUDA(cudaLaunchCooperativeKernel((const void *)jcg_kernel, dim3(c->jcg_grid),
                                       dim3(kThreads), args, 0, c->stream));
  c->launches++;
  return ADC_OK;
}

int launch_jcg(adc_ctx *c, int eta_update) { return launch_jcg_impl(c, eta_update, 0, 1); }

}  // namespace adc
