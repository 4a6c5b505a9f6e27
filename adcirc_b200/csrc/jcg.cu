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
#include "tma.cuh"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>
#include <type_traits>

namespace adc {

// 32-byte node record (dtwd, d, d_prev, -) moved with one 256-bit access.
struct __align__(32) P4 {
  double x, y, z, w;
};

__device__ __forceinline__ P4 ld_p4(const P4 *p) {
  P4 r;
  asm volatile("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];"
               : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w)
               : "l"(p));
  return r;
}

__device__ __forceinline__ void st_p4(P4 *p, double x, double y, double z, double w) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(x), "d"(y), "d"(z), "d"(w)
               : "memory");
}

struct JcgArgs {
  int n, nslices, nrb, itmax;
  const int *sl_ptr, *sl_w, *col, *rlen;
  double *offd, *soff, *diag, *rhs;
  float *soff32;                // FP32 copy of the scaled matrix (mixed mode)
  double *u, *u1, *w;
  P4 *p0, *p1;
  double *part, *tri;
  Itp *itp;
  Bar *bar;
  void *arrive;             // ArriveLine[nrb + 1]: the row blocks' and the scalar block's
  Flags *flags;
  int eta_update;
  int do_peror;
  // resident variant
  int rows_max;               // rows of the largest row block
  int halo_max;               // halo nodes of the largest row block
  int stage_bytes;            // one staged slice: local columns + values
  int stage_wcap;             // widest slice that is staged; wider ones are read in place
  const unsigned short *lcol; // per slot: block-local value index
  const int *halo_ptr;        // [nrb + 1] into halo_ids
  const int *halo_ids;        // halo nodes of each row block (global rows)
  const unsigned char *exp;   // per row: read by another row block
  int defer_drift;            // 1: leave the COEF unscal drift to the next step;
                              // 2: drop it (mixed mode, COEF is rebuilt or kept as is)
  int *drift_pending;         // set to 1 when the drift is left pending
  const int *nodecode;
  const double *eta1;
  double *eta2;
};

__device__ __forceinline__ double vld(const double *p) { return *(const volatile double *)p; }

// ---------------------------------------------------------------- barrier
// Contention-free flag barrier that carries its data, read by every block.
// Each block owns one 128-byte arrival line of four slots, used in turn by
// the barrier generations (slot g & 3); a row block posts its three partial
// sums there, the scalar block (the last block of the grid) posts the
// eigenvalue estimate cme that its chgcon produced for this barrier.  An
// empty word holds kEmpty, a signalling-NaN bit pattern no arithmetic
// produces.  Every block polls all arrival lines until each word of the
// current slot is filled, sums the row blocks' partials in one fixed order
// (the same in every block, so every block holds the same bits) and runs
// the serial ITPACK step (pstop_nrms, parcon) itself on its own copy of the
// ITPACK scalars: one L2 round trip both signals and delivers, and no
// release step follows.  A block empties its own slot (g + 2) & 3 when it
// posts generation g: every reader of generation g - 2 has finished
// reading before any block can post generation g (it first had to see
// everyone's generation g - 1 arrival).  Every word is an aligned 8-byte
// access (single-copy atomic); waits are bounded.
constexpr unsigned long long kEmpty = 0x7FF4DEADBEEF0001ull;

struct alignas(128) ArriveLine {
  unsigned long long slot[4][4];   // (p0, p1, p2, -) of a row block; (cme, 0, 0, -) of the scalar block
};

__device__ __forceinline__ unsigned long long dbits(double x) {
  return (unsigned long long)__double_as_longlong(x);
}
__device__ __forceinline__ double bitsd(unsigned long long u) {
  return __longlong_as_double((long long)u);
}

// Release/acquire fence at GPU scope: orders a block's results before the
// barrier words it writes, and the words it polled before what it reads next.
__device__ __forceinline__ void fence_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Polls N words until all are filled; v receives them.  Bounded.
template <int N>
__device__ bool poll_full(volatile unsigned long long *p, unsigned long long (&v)[N],
                          Flags *flags) {
  const long long t0 = clock64();
  for (;;) {
    bool full = true;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      v[k] = p[k];
      full = full && (v[k] != kEmpty);
    }
    if (full) return true;
    if (*(volatile int *)&flags->timeout) return false;
    if (clock64() - t0 > kSpinCycles) {
      atomicExch(&flags->timeout, 1);
      return false;
    }
  }
}

__device__ Rec read_rec(const Rec *r) {
  const volatile Rec *v = r;
  Rec o;
  o.c1 = v->c1;
  o.c2 = v->c2;
  o.c3 = v->c3;
  o.c4 = v->c4;
  o.halt = v->halt;
  o.need_unorm = v->need_unorm;
  o.in = v->in;
  o.pad_ = 0;
  return o;
}

// The record's integers in one word (never kEmpty: the top 16 bits are 0).
__device__ __forceinline__ unsigned long long pack_rec(const Rec &r) {
  return (unsigned long long)(unsigned)r.in | ((unsigned long long)(r.halt & 0xff) << 32) |
         ((unsigned long long)(r.need_unorm & 0xff) << 40);
}

// Serial ITPACK state of one solve, held in registers of the scalar block's
// thread 0 (echall/itjcg/chgcon/pstop/parcon variables).
struct ItpLocal {
  double zeta, cme, gamma, rho, gamold, rhoold, delnnm, delsnm, udnm, stptst, cmold, rparm1;
  int itmax, adapt, q1, isym, chg_ier;
};

// ---------------------------------------------------------------- scalars
// determ (itpackv.F:1029-1068): the three-term recurrence for
// det(tri - x I), evaluated with the two trailing values in registers
// (same operations, same order as the wk1/wk2 arrays of the reference).
// tri(i,1) = t1[i-1], tri(i,2) = t2[i-1], held in shared memory.
__device__ double determ_d(int n, const double *t1, const double *t2, double xlmda) {
  double w2 = t1[n - 1] - xlmda;                       // wk2(n)
  double w1 = (t1[n - 2] - xlmda) * w2 + t2[n - 1];    // wk2(n-1)
  for (int l = n - 2; l >= 1; --l) {
    double w = (t1[l - 1] - xlmda) * w1 + t2[l] * w2;  // wk2(l)
    w2 = w1;
    w1 = w;
  }
  return w1;
}

// zbrent (itpackv.F:2521-2781): Brent root of the characteristic
// polynomial of the CG tridiagonal on [a, b].
__device__ void zbrent_d(int n, const double *t1, const double *t2, double eps, double t,
                         double &a, double &b, int &maxfn, int &ier) {
  double c = 0, d = 0, e = 0, p, q, r, s, fa, fb, fc, tol, rm, rone, temp;
  ier = 0;
  int ic = 2;
  fa = determ_d(n, t1, t2, a);
  fb = determ_d(n, t1, t2, b);
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
    fb = determ_d(n, t1, t2, s);
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

// chgcon, jacobi case (itpackv.F:893-1027), for iteration `in`.  The
// tridiagonal lives in the scalar block's shared memory (t1, t2).
__device__ void chgcon_d(ItpLocal *it, double *t1, double *t2, int in) {
  double start = it->cme, end1 = 0.0;
  int ip = in;
  if (ip == 0) {
    it->cmold = 0.0;
    it->cme = 0.0;
    return;
  }
  if (ip == 1) {
    end1 = 1.0 - 1.0 / it->gamma;
    t1[0] = end1;
    t2[0] = 0.0;
    it->cme = end1;
    return;
  }
  if (fabs(start - it->cmold) <= it->zeta * start) {
    it->adapt = 0;
    return;
  }
  it->cmold = start;
  t1[ip - 1] = 1.0 - 1.0 / it->gamma;
  t2[ip - 1] = (1.0 - it->rho) / (it->rho * it->rhoold * it->gamma * it->gamold);
  int ier = 0;
  if (it->isym != 0) {
    ier = 903;
  } else {
    int nsig = nsig_of(it->zeta);
    int maxfn = it->itmax > 50 ? it->itmax : 50;
    double a = start, b = 1.0;
    zbrent_d(ip, t1, t2, 0.0, pow10_neg(nsig), a, b, maxfn, ier);
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
__device__ int pstop_d(ItpLocal *it, int in, double unrm, double dnrm) {
  double con = it->cme, uold, tr, tl;
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
  if (tl >= tr * it->zeta) return 0;
  return 1;
}

// parcon (itpackv.F:1774-1851) for iteration `in`.
__device__ void parcon_d(ItpLocal *it, int in, double dtnrm, double c[4]) {
  double rhoold = it->rho;
  double gamold = it->gamma;
  it->gamma = 1.0 / (1.0 - dtnrm / it->delnnm);
  it->rho = 1.0;
  if (in != 0) it->rho = 1.0 / (1.0 - it->gamma * it->delnnm / (gamold * it->delsnm * rhoold));
  it->delsnm = it->delnnm;
  it->gamold = gamold;
  it->rhoold = rhoold;
  c[0] = it->rho * it->gamma;
  c[1] = it->rho;
  c[2] = 1.0 - it->rho;
  c[3] = it->rho * (1.0 - it->gamma);
}

// ------------------------------------------------------------ row access
// A row's off-diagonal slots are processed in chunks of kCh: the column and
// value of every slot of the chunk are loaded first, then all neighbour
// values are gathered, so the loads of a chunk are in flight together.
// Accumulation keeps the slot order (pjac's j order).
constexpr int kCh = 6;
constexpr int kRowUnroll = 8;   // rows per thread whose loads issue together
constexpr int kHaloPre = 2;     // halo records per thread fetched ahead of the row update

// L2 prefetch of the next slice of a warp: the column and value rows of its
// slots and its own-row vector entries, one 128-byte line per lane.
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ void prefetch_slice(int lane, int ptr, int w, int row0, const int *col,
                                               const double *val, const P4 *pv,
                                               const double *u0, const double *u1) {
  // lines: col w, val 2w, pv 8, u0 2, u1 2
  const int ncol = w, nval = 2 * w;
  for (int l = lane; l < ncol + nval + 12; l += 32) {
    const char *a;
    if (l < ncol) a = (const char *)(col + ptr) + 128 * l;
    else if (l < ncol + nval) a = (const char *)(val + ptr) + 128 * (l - ncol);
    else if (l < ncol + nval + 8) a = (const char *)(pv + row0) + 128 * (l - ncol - nval);
    else if (l < ncol + nval + 10) a = (const char *)(u0 + row0) + 128 * (l - ncol - nval - 8);
    else a = (const char *)(u1 + row0) + 128 * (l - ncol - nval - 10);
    prefetch_l2(a);
  }
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

// One barrier of generation g for every block.  Row blocks post their
// block sums of (p0, p1, p2), the scalar block posts `cme`; then every block
// gathers the row blocks' posts in block order (thread t takes blocks t,
// t + blockDim, ...; then a fixed tree) and thread 0 runs
// `serial(s0, s1, s2, cme)`.  Returns false on timeout.
template <class F>
__device__ bool grid_phase(const JcgArgs &a, bool scalar_block, unsigned g, double p0, double p1,
                           double p2, double cme, F serial) {
  __shared__ int bad;
  __shared__ double s_cme;
  const int sl = g & 3, sl_old = (g + 2) & 3;
  if (!scalar_block) block_sum3(p0, p1, p2);
  if (threadIdx.x == 0) {
    bad = 0;
    volatile unsigned long long *own = ((ArriveLine *)a.arrive + blockIdx.x)->slot[0];
    own[4 * sl_old + 0] = kEmpty;
    own[4 * sl_old + 1] = kEmpty;
    own[4 * sl_old + 2] = kEmpty;
    fence_gpu();   // the block's results (and the emptied slot) before its arrival
    if (scalar_block) {
      own[4 * sl + 0] = dbits(cme);
      own[4 * sl + 1] = 0ull;
      own[4 * sl + 2] = 0ull;
    } else {
      own[4 * sl + 0] = dbits(p0);
      own[4 * sl + 1] = dbits(p1);
      own[4 * sl + 2] = dbits(p2);
    }
  }
  __syncthreads();
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int b = threadIdx.x; b <= a.nrb; b += blockDim.x) {
    volatile unsigned long long *ap = ((ArriveLine *)a.arrive + b)->slot[sl];
    unsigned long long v[3];
    if (!poll_full<3>(ap, v, a.flags)) {
      bad = 1;
      break;
    }
    if (b == a.nrb) {
      s_cme = bitsd(v[0]);
    } else {
      s0 += bitsd(v[0]);
      s1 += bitsd(v[1]);
      s2 += bitsd(v[2]);
    }
  }
  fence_gpu();
  __syncthreads();
  if (bad) return false;
  block_sum3(s0, s1, s2);
  if (threadIdx.x == 0) serial(s0, s1, s2, s_cme);
  __syncthreads();
  return true;
}

// Reducing phase end: `serial(s0, s1, s2, cme)` runs in every block on the
// same sums.
template <class F>
__device__ bool phase_reduce(const JcgArgs &a, bool scalar_block, unsigned &g, double p0,
                             double p1, double p2, double cme, F serial) {
  ++g;
  return grid_phase(a, scalar_block, g, p0, p1, p2, cme, serial);
}

// Plain barrier (no partials, no record).
__device__ bool phase_sync(const JcgArgs &a, bool scalar_block, unsigned &g) {
  ++g;
  return grid_phase(a, scalar_block, g, 0.0, 0.0, 0.0, 0.0, [](double, double, double, double) {});
}


// Per-warp double-buffered bulk copies of whole slices (block-local
// columns + one value array) into shared memory, for the resident variant.
// Every copy that is issued is waited for before the next phase.
struct SlicePipe {
  unsigned char *stg0;        // this warp's two buffers
  uint64_t *bar0;             // and their mbarriers
  const int2 *meta;           // per slice of the block: (first slot, width)
  const unsigned short *lcol;
  Flags *flags;
  int stage_bytes, s0, s1, first, step, lane;
  uint32_t parbits;
  int wcap;                   // slices wider than this are not staged

  __device__ bool staged(int sl) const { return meta[sl - s0].y <= wcap; }

  // V: the staged value type (FP64 matrix, or FP32 in the mixed mode)
  template <class V>
  __device__ void issue(int sl, int st, const V *vals) {
    if (lane == 0 && staged(sl)) {
      const int2 mt = meta[sl - s0];
      const uint32_t w = (uint32_t)mt.y;
      const uint32_t vb = w * 32u * (uint32_t)sizeof(V);
      unsigned char *b = stg0 + (size_t)st * stage_bytes;
      mbar_expect_tx(bar0 + st, w * 64u + vb);
      if (w > 0) {
        bulk_load(b, lcol + mt.x, w * 64u, bar0 + st);
        bulk_load(b + w * 64u, vals + mt.x, vb, bar0 + st);
      }
    }
  }
  // Starts the warp's first two slices; with `fence`, first orders earlier
  // generic writes of `vals` before the copies.
  template <class V>
  __device__ void begin(const V *vals, bool fence) {
    if (fence && lane == 0) fence_proxy_async_all();
    if (first < s1) issue(first, 0, vals);
    if (first + step < s1) issue(first + step, 1, vals);
  }
  __device__ bool wait(int st, bool other_in_flight) {
    long long tw = clock64();
    while (!mbar_try_wait(bar0 + st, (parbits >> st) & 1u)) {
      if (clock64() - tw > kSpinCycles) {
        if (lane == 0) {
          atomicExch(&flags->timeout, 1);
          // let the copy already issued into the other buffer land
          if (other_in_flight) {
            long long t1w = clock64();
            while (!mbar_try_wait(bar0 + (st ^ 1), (parbits >> (st ^ 1)) & 1u) &&
                   clock64() - t1w < kSpinCycles) {
            }
          }
        }
        __syncwarp();
        return false;
      }
    }
    parbits ^= 1u << st;
    return true;
  }
  // body(sl, lc, lv): one slice from shared memory (or, for a slice wider
  // than wcap, in place from global memory, which has the same layout);
  // lc/lv hold slot q of lane l at [q * 32 + l].  Returns false on an
  // expired wait.
  template <class V, class F>
  __device__ bool run(const V *vals, F body) {
    int k = 0;
    for (int sl = first; sl < s1; sl += step, ++k) {
      const int st = k & 1;
      const int2 mt = meta[sl - s0];
      if (mt.y > wcap) {
        body(sl, lcol + mt.x, vals + mt.x);
      } else {
        if (!wait(st, sl + step < s1 && staged(sl + step))) return false;
        const unsigned char *b = stg0 + (size_t)st * stage_bytes;
        body(sl, (const unsigned short *)b, (const V *)(b + (size_t)mt.y * 64));
      }
      __syncwarp();
      if (sl + 2 * step < s1) issue(sl + 2 * step, st, vals);
    }
    return true;
  }
};

// ------------------------------------------------------------ the kernel
// kRes: 1 = resident variant.  VT: storage type of the scaled matrix the
// iterations stream (double; float in the mixed-precision mode, where the
// products still accumulate in FP64).
template <int kRes, class VT>
__global__ void __launch_bounds__(kThreads, 2) jcg_kernel(JcgArgs a) {
  griddep_wait();
  VT *const sv_store = std::is_same<VT, float>::value ? (VT *)a.soff32 : (VT *)a.soff;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const bool scalar_block = (blockIdx.x == (unsigned)a.nrb);
  const int s0 = scalar_block ? 0 : (int)((long long)a.nslices * blockIdx.x / a.nrb);
  const int s1 = scalar_block ? 0 : (int)((long long)a.nslices * (blockIdx.x + 1) / a.nrb);
  const int n = a.n;
  const int r0 = s0 * kSlice, rows = (s1 - s0) * kSlice;   // the block's rows [r0, r0 + rows)
  extern __shared__ __align__(128) unsigned char s_dyn[];
  // Dynamic shared memory.  Scalar block: tri(:,1) and tri(:,2).  Row blocks
  // of the resident variant: dtwd of the block's rows; two value buffers
  // (d of the rows, then the halo's new d) that trade roles every
  // iteration; per row its length and export bit; the slice table; one
  // mbarrier and two staging buffers per warp.
  double *t1 = (double *)s_dyn, *t2 = t1 + a.itmax + 1;
  const int RB = a.rows_max, VB = a.rows_max + a.halo_max;
  double *S_t = (double *)s_dyn;
  double *S_dd = S_t + RB;
  unsigned char *S_le = (unsigned char *)(S_dd + 2 * VB);
  int2 *S_meta = (int2 *)(S_le + ((RB + 127) & ~127));
  int *S_hid = (int *)(S_meta + ((RB / kSlice + 15) & ~15));   // the block's halo nodes
  uint64_t *S_bar = (uint64_t *)(S_hid + ((a.halo_max + 31) & ~31));
  unsigned char *S_stage = (unsigned char *)(S_bar + 16);
  const int nhalo = (kRes && !scalar_block) ? a.halo_ptr[blockIdx.x + 1] - a.halo_ptr[blockIdx.x] : 0;
  SlicePipe pipe{S_stage + (size_t)(2 * warp) * a.stage_bytes, &S_bar[2 * warp], S_meta, a.lcol,
                 a.flags, a.stage_bytes, s0, s1, s0 + warp, nwarps, lane, 0u, a.stage_wcap};
  Rec *rec = &a.itp->rec;
  __shared__ ItpLocal L;              // used by the scalar block's thread 0 only
  __shared__ Rec s_rec;               // the record of the last reducing barrier
  unsigned gen = 0;                   // barrier generation within this launch
  if (threadIdx.x == 0) {   // every block steps its own copy of the ITPACK scalars
    const volatile Itp *g = a.itp;
    L.zeta = g->zeta; L.cme = g->cme; L.gamma = g->gamma; L.rho = g->rho;
    L.gamold = g->gamold; L.rhoold = g->rhoold; L.delnnm = g->delnnm; L.delsnm = g->delsnm;
    L.udnm = g->udnm; L.stptst = g->stptst; L.cmold = g->cmold; L.rparm1 = g->rparm1;
    L.itmax = g->itmax; L.adapt = g->adapt; L.q1 = g->q1; L.isym = g->isym; L.chg_ier = 0;
  }

  // P2 needs the unorm flag of iteration 0, set before the launch.
  Rec r = read_rec(rec);
  const int need_u0 = r.need_unorm;
  double pd = 0.0, pt = 0.0, pu = 0.0;
  if (!kRes) {
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
      }
    }
    if (!phase_sync(a, scalar_block, gen)) return;

    // P1: scaled off-diagonals, the reference's unscal drift of the resident
    // matrix, and the initial pseudo-residual d0 = pjac(u') + rhs' - u'.
    for (int s = s0 + warp; s < s1; s += nwarps) {
      int i = s * kSlice + lane;
      if (i < n) {
        int len = a.rlen[i];
        int base = a.sl_ptr[s] + lane;
        double wi = a.w[i];
        double ui = a.u[i];
        double winv_i = 1.0 / wi;
        double acc = a.rhs[i];
        for (int c0 = 0; c0 < len; c0 += kCh) {
          int jj[kCh];
          double vo[kCh], wj[kCh], uj[kCh];
  #pragma unroll
          for (int k = 0; k < kCh; ++k)
            if (c0 + k < len) {
              int idx = base + (c0 + k) * kSlice;
              jj[k] = a.col[idx];
              vo[k] = a.offd[idx];
            }
  #pragma unroll
          for (int k = 0; k < kCh; ++k)
            if (c0 + k < len) {
              wj[k] = a.w[jj[k]];
              uj[k] = a.u[jj[k]];
            }
  #pragma unroll
          for (int k = 0; k < kCh; ++k)
            if (c0 + k < len) {
              int idx = base + (c0 + k) * kSlice;
              double sv = vo[k] * wi * wj[k];
              a.soff[idx] = sv;
              if (!a.defer_drift) a.offd[idx] = sv * winv_i * (1.0 / wj[k]);
              acc = acc - sv * uj[k];
            }
        }
        st_p4(a.p0 + i, 0.0, acc - ui, 0.0, 0.0);   // (dtwd0 later, d0, d(-1) = 0)
        a.diag[i] = winv_i * winv_i;
      }
    }
    if (!phase_sync(a, scalar_block, gen)) return;

    // P2: dtwd0 = -A' d0 and the iteration-0 norms; the scalar block runs
    // chgcon for in = 0 (ip = 0: cme = 0) while the rows work.
    {
      for (int s = s0 + warp; s < s1; s += nwarps) {
        int i = s * kSlice + lane;
        if (i < n) {
          int len = a.rlen[i];
          int base = a.sl_ptr[s] + lane;
          double acc = 0.0;
          for (int c0 = 0; c0 < len; c0 += kCh) {
            int jj[kCh];
            double vv[kCh], xx[kCh];
  #pragma unroll
            for (int k = 0; k < kCh; ++k)
              if (c0 + k < len) {
                int idx = base + (c0 + k) * kSlice;
                jj[k] = a.col[idx];
                vv[k] = a.soff[idx];
              }
  #pragma unroll
            for (int k = 0; k < kCh; ++k)
              if (c0 + k < len) xx[k] = a.p0[jj[k]].y;
  #pragma unroll
            for (int k = 0; k < kCh; ++k)
              if (c0 + k < len) acc = acc - vv[k] * xx[k];
          }
          a.p0[i].x = acc;
          double di = a.p0[i].y;
          pd += di * di;
          pt += di * acc;
          if (need_u0) { double ui = a.u[i]; pu += ui * ui; }
        }
      }
    }
  } else {
    // Resident prologue.  Shared memory first holds, per row of the block
    // and per halo node, w = 1/sqrt(diag) and u' (P1), then d0 (P2).
    double *Uv = S_dd, *Wv = S_dd + VB;
    if (!scalar_block) {
      // Everything the prologue needs from global memory is requested
      // before any of it is stored, so the loads share one round trip: the
      // slice table, the halo list, and per row its length, export bit and
      // the diagonal, u and rhs of P0 (scal part 1: u' = u*sqrt(d),
      // w = 1/sqrt(d), rhs' = rhs*w).
      const int nsl = s1 - s0;
      const int h0 = a.halo_ptr[blockIdx.x];
      int2 mt = make_int2(0, 0);
      if ((int)threadIdx.x < nsl) mt = make_int2(a.sl_ptr[s0 + threadIdx.x], a.sl_w[s0 + threadIdx.x]);
      int hid[kHaloPre];
#pragma unroll
      for (int k = 0; k < kHaloPre; ++k) {
        const int h = threadIdx.x + k * blockDim.x;
        hid[k] = h < nhalo ? a.halo_ids[h0 + h] : 0;
      }
      for (int base = threadIdx.x; base < rows; base += kRowUnroll * blockDim.x) {
        double dg[kRowUnroll], uu[kRowUnroll], rh[kRowUnroll];
        int rl[kRowUnroll];
        unsigned char ex[kRowUnroll];
#pragma unroll
        for (int k = 0; k < kRowUnroll; ++k) {
          const int idx = base + k * blockDim.x, i = r0 + idx;
          if (idx < rows && i < n) {
            dg[k] = a.diag[i]; uu[k] = a.u[i]; rh[k] = a.rhs[i];
            rl[k] = a.rlen[i]; ex[k] = a.exp[i];
          }
        }
#pragma unroll
        for (int k = 0; k < kRowUnroll; ++k) {
          const int idx = base + k * blockDim.x, i = r0 + idx;
          if (idx < rows) S_le[idx] = i < n ? (unsigned char)(rl[k] | (ex[k] ? 128 : 0)) : 0;
          if (idx < rows && i < n) {
            double work = sqrt(dg[k]);
            const double up = uu[k] * work;
            double wv = 1.0 / work;
            a.u1[i] = up;   // u' goes to u1: u keeps the raw guess until P2
            a.w[i] = wv;
            a.rhs[i] = rh[k] * wv;
            Uv[idx] = up;
            Wv[idx] = wv;
            if (need_u0) pu += up * up;
          }
        }
      }
      if ((int)threadIdx.x < nsl) S_meta[threadIdx.x] = mt;
      for (int k = threadIdx.x + blockDim.x; k < nsl; k += blockDim.x)
        S_meta[k] = make_int2(a.sl_ptr[s0 + k], a.sl_w[s0 + k]);
#pragma unroll
      for (int k = 0; k < kHaloPre; ++k) {
        const int h = threadIdx.x + k * blockDim.x;
        if (h < nhalo) S_hid[h] = hid[k];
      }
      for (int h = threadIdx.x + kHaloPre * blockDim.x; h < nhalo; h += blockDim.x)
        S_hid[h] = a.halo_ids[h0 + h];
      if (threadIdx.x < 2 * nwarps) mbar_init(&S_bar[threadIdx.x], 1);
      mbar_fence_init();
    }
    // No grid barrier after P0: P1 reads only this block's own P0 results,
    // and forms the halo's u' and w itself from the raw u and diag, which
    // no block overwrites before P2.
    __syncthreads();
    // P1: scaled off-diagonals, the reference's unscal drift of the resident
    // matrix, and d0 = pjac(u') + rhs' - u' (kept in S_t until P2).
    if (!scalar_block) {
      pipe.begin(a.offd, false);   // offd was last written by an earlier kernel
      const int nh = nhalo;
      for (int h = threadIdx.x; h < nh; h += blockDim.x) {
        const int j = S_hid[h];
        double work = sqrt(a.diag[j]);   // the owner's P0 expressions
        Uv[RB + h] = a.u[j] * work;
        Wv[RB + h] = 1.0 / work;
      }
      __syncthreads();
      bool ok = pipe.run(a.offd, [&](int sl, const unsigned short *lc, const double *lv) {
        const int i = sl * kSlice + lane, idx = i - r0;
        if (i < n) {
          const int len = S_le[idx] & 127;
          const int base = S_meta[sl - s0].x + lane;
          const double wi = Wv[idx], ui = Uv[idx];
          const double winv_i = 1.0 / wi;
          double acc = a.rhs[i];
          for (int q = 0; q < len; ++q) {
            const int lq = lc[q * kSlice + lane];
            const double wj = Wv[lq];
            const double sv = lv[q * kSlice + lane] * wi * wj;
            sv_store[base + q * kSlice] = (VT)sv;
            if (!a.defer_drift) a.offd[base + q * kSlice] = sv * winv_i * (1.0 / wj);
            acc = acc - sv * Uv[lq];
          }
          const double d0 = acc - ui;
          if (S_le[idx] & 128) st_p4(a.p0 + i, 0.0, d0, 0.0, 0.0);
          S_t[idx] = d0;
        }
      });
      if (!ok) atomicExch(&a.flags->timeout, 1);
      fence_proxy_async_all();   // soff is read by bulk copies from here on
    }
    if (!phase_sync(a, scalar_block, gen)) return;
    // P2: dtwd0 = -A' d0 and the iteration-0 norms.
    if (!scalar_block) {
      pipe.begin((const VT *)sv_store, true);   // the scaled matrix was just written
      double *Dv = S_dd;
      for (int idx = threadIdx.x; idx < rows; idx += blockDim.x) {
        Dv[idx] = S_t[idx];
        S_dd[VB + idx] = 0.0;   // d(-1)
        const int i = r0 + idx;
        if (i < n) {
          // every block has read the raw u and diag by now (the P1 barrier)
          a.u[i] = 0.0;   // u(-1) of the recurrence
          const double winv_i = 1.0 / a.w[i];
          a.diag[i] = winv_i * winv_i;   // scal/unscal of the diagonal
        }
      }
      const int nh = nhalo;
      for (int h = threadIdx.x; h < nh; h += blockDim.x) Dv[RB + h] = a.p0[S_hid[h]].y;
      __syncthreads();
      bool ok = pipe.run((const VT *)sv_store, [&](int sl, const unsigned short *lc, const VT *lv) {
        const int i = sl * kSlice + lane, idx = i - r0;
        if (i < n) {
          const int len = S_le[idx] & 127;
          double acc = 0.0;
          for (int q = 0; q < len; ++q)
            acc = acc - (double)lv[q * kSlice + lane] * Dv[lc[q * kSlice + lane]];
          if (S_le[idx] & 128) a.p0[i].x = acc;
          S_t[idx] = acc;
          const double di = Dv[idx];
          pd += di * di;
          pt += di * acc;
        }
      });
      if (!ok) atomicExch(&a.flags->timeout, 1);
    }
  }
  {
    if (scalar_block && threadIdx.x == 0 && L.adapt) chgcon_d(&L, t1, t2, 0);
    const int need_u = need_u0;
    bool ok = phase_reduce(a, scalar_block, gen, pd, pt, pu, L.cme,
                           [&](double sd, double st, double su, double cme) {
      L.cme = cme;   // chgcon's estimate, from the scalar block
      L.delnnm = sd;
      int halt = pstop_d(&L, 0, need_u ? su : 1.0, sd);
      double c[4] = {0, 0, 0, 0};
      if (!halt) {
        if (L.itmax == 0) halt = 2;
        else parcon_d(&L, 0, st, c);
      }
      Rec *vr = &s_rec;
      vr->c1 = c[0]; vr->c2 = c[1]; vr->c3 = c[2]; vr->c4 = c[3];
      vr->halt = halt;
      vr->need_unorm = !(L.q1 || ((1 > 5) && (1 % 5 != 0)));
      vr->in = 0;
    });
    if (!ok) return;
  }

  // Iteration phases: phase `in` forms u(in+1), d(in+1), dtwd(in+1) and the
  // norms of iteration in+1.  P[in % 2][i] = (dtwd(in), d(in), d(in-1)) so
  // a neighbour's three values arrive in one 32-byte sector.
  P4 *P[2] = {a.p0, a.p1};
  // u(in) and u(in-1): the resident prologue leaves u' in u1 and zeroes u
  double *U[2] = {kRes ? a.u1 : a.u, kRes ? a.u : a.u1};
  int cur = 0;   // resident variant: S_dd half holding d(in)
  for (int in = 0; in < a.itmax; ++in) {
    r = s_rec;
    if (r.halt) break;
    const double c1 = r.c1, c2 = r.c2, c3 = r.c3, c4 = r.c4;
    const int need_u = r.need_unorm;
    const P4 *pc = P[in % 2];
    P4 *pn = P[(in + 1) % 2];
    const double *uc = U[in % 2];
    double *un = U[(in + 1) % 2];
    double pd = 0.0, pt = 0.0, pu = 0.0;
    if (!kRes) {
      for (int s = s0 + warp; s < s1; s += nwarps) {
        int i = s * kSlice + lane;
        const int sn = s + nwarps;
        if (sn < s1)
          prefetch_slice(lane, a.sl_ptr[sn], a.sl_w[sn], sn * kSlice, a.col, a.soff, pc, uc, un);
        if (i < n) {
          const P4 me = ld_p4(pc + i);
          double unew = c1 * me.y + c2 * uc[i] + c3 * un[i];
          double dnew = c1 * me.x + c4 * me.y + c3 * me.z;
          int len = a.rlen[i];
          int base = a.sl_ptr[s] + lane;
          double acc = 0.0;
          for (int c0 = 0; c0 < len; c0 += kCh) {
            int jj[kCh];
            double vv[kCh];
            P4 xx[kCh];
  #pragma unroll
            for (int k = 0; k < kCh; ++k)
              if (c0 + k < len) {
                int idx = base + (c0 + k) * kSlice;
                jj[k] = a.col[idx];
                vv[k] = a.soff[idx];
              }
  #pragma unroll
            for (int k = 0; k < kCh; ++k)
              if (c0 + k < len) xx[k] = ld_p4(pc + jj[k]);
  #pragma unroll
            for (int k = 0; k < kCh; ++k)
              if (c0 + k < len) {
                double dj = c1 * xx[k].x + c4 * xx[k].y + c3 * xx[k].z;
                acc = acc - vv[k] * dj;
              }
          }
          un[i] = unew;
          st_p4(pn + i, acc, dnew, me.y, 0.0);
          pd += dnew * dnew;
          pt += dnew * acc;
          if (need_u) pu += unew * unew;
        }
      }
    } else if (!scalar_block) {
      // Resident variant.  The warp's first two slices start streaming
      // before phase A.
      pipe.begin((const VT *)sv_store, false);   // unchanged since P2's fence
      // Phase A: the 3-term update of the block's rows, d(in+1) written
      // over d(in-1); then the new d of the halo nodes from their owners'
      // exported records (same expression, same bits).
      double *Sd = S_dd + cur * VB, *Sdn = S_dd + (cur ^ 1) * VB;
      const int nh = nhalo;
      P4 hv[kHaloPre];   // the first halo records, loaded with the rows' vectors
#pragma unroll
      for (int k = 0; k < kHaloPre; ++k) {
        const int h = threadIdx.x + k * blockDim.x;
        if (h < nh) hv[k] = ld_p4(pc + S_hid[h]);
      }
      for (int base = threadIdx.x; base < rows; base += kRowUnroll * blockDim.x) {
        double ucv[kRowUnroll], unv[kRowUnroll];
#pragma unroll
        for (int k = 0; k < kRowUnroll; ++k) {
          const int idx = base + k * blockDim.x, i = r0 + idx;
          if (idx < rows && i < n) { ucv[k] = uc[i]; unv[k] = un[i]; }
        }
#pragma unroll
        for (int k = 0; k < kRowUnroll; ++k) {
          const int idx = base + k * blockDim.x, i = r0 + idx;
          if (idx < rows && i < n) {
            const double dn = c1 * S_t[idx] + c4 * Sd[idx] + c3 * Sdn[idx];
            const double unew = c1 * Sd[idx] + c2 * ucv[k] + c3 * unv[k];
            Sdn[idx] = dn;
            un[i] = unew;
            if (need_u) pu += unew * unew;
          }
        }
      }
#pragma unroll
      for (int k = 0; k < kHaloPre; ++k) {
        const int h = threadIdx.x + k * blockDim.x;
        if (h < nh) Sdn[RB + h] = c1 * hv[k].x + c4 * hv[k].y + c3 * hv[k].z;
      }
      for (int h = threadIdx.x + kHaloPre * blockDim.x; h < nh; h += blockDim.x) {
        const P4 o = ld_p4(pc + S_hid[h]);
        Sdn[RB + h] = c1 * o.x + c4 * o.y + c3 * o.z;
      }
      __syncthreads();
      // Phase B: the SpMV from shared memory, slot order as in pjac.
      bool ok = pipe.run((const VT *)sv_store, [&](int sl, const unsigned short *lc, const VT *lv) {
        const int i = sl * kSlice + lane, idx = i - r0;
        if (i < n) {
          const unsigned le = S_le[idx];
          const int len = (int)(le & 127u);
          double acc = 0.0;
#pragma unroll 4
          for (int q = 0; q < len; ++q)
            acc = acc - (double)lv[q * kSlice + lane] * Sdn[lc[q * kSlice + lane]];
          const double dn = Sdn[idx];
          if (le & 128u) st_p4(pn + i, acc, dn, Sd[idx], 0.0);
          S_t[idx] = acc;
          pd += dn * dn;
          pt += dn * acc;
        }
      });
      if (!ok) atomicExch(&a.flags->timeout, 1);
      cur ^= 1;
    }
    const int m = in + 1;
    if (scalar_block && threadIdx.x == 0 && L.adapt) chgcon_d(&L, t1, t2, m);
    bool ok = phase_reduce(a, scalar_block, gen, pd, pt, pu, L.cme,
                           [&](double sd, double st, double su, double cme) {
      L.cme = cme;   // chgcon's estimate, from the scalar block
      L.delnnm = sd;
      int halt = pstop_d(&L, m, need_u ? su : 1.0, sd);
      double c[4] = {0, 0, 0, 0};
      if (!halt) {
        if (m >= L.itmax) halt = 2;
        else parcon_d(&L, m, st, c);
      }
      int mm = m + 1;
      Rec *vr = &s_rec;
      vr->c1 = c[0]; vr->c2 = c[1]; vr->c3 = c[2]; vr->c4 = c[3];
      vr->halt = halt;
      vr->need_unorm = !(L.q1 || ((mm > 5) && (mm % 5 != 0)));
      vr->in = m;
    });
    if (!ok) return;
  }
  r = s_rec;
  const int fin = r.in;
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
          cc = cc - (double)sv_store[idx] * usol[a.col[idx]];
        }
        double wk2 = (a.rhs[i] - cc) / wv;
        pr += wk2 * wk2;
      }
    }
    bool ok = phase_reduce(a, scalar_block, gen, pb, pr, 0.0, 0.0,
                           [&](double sb, double sr, double, double) {
      if (scalar_block) {
        a.itp->dtnrm = sb;
        a.itp->unorm = sr;
      }
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
  if (scalar_block && threadIdx.x == 0) {
    int h = r.halt;
    if (h == 2) L.rparm1 = L.stptst;   // itpackv.F:394
    volatile Itp *g = a.itp;
    g->zeta = L.zeta; g->cme = L.cme; g->gamma = L.gamma; g->rho = L.rho;
    g->gamold = L.gamold; g->rhoold = L.rhoold; g->delnnm = L.delnnm; g->delsnm = L.delsnm;
    g->udnm = L.udnm; g->stptst = L.stptst; g->cmold = L.cmold; g->rparm1 = L.rparm1;
    g->adapt = L.adapt; g->q1 = L.q1; g->chg_ier = L.chg_ier;
    g->in = fin;
    g->halt = h;
    if (a.defer_drift == 1) *a.drift_pending = 1;
    a.flags->numitr = fin;
    a.flags->ier = (h == 2) ? 13 : 0;
    a.flags->zeta = L.rparm1;
    a.flags->cme = L.cme;
  }
}

// Per-solve ITPACK initialisation (echall, itpackv.F:1212-1255, plus the
// zeta floor of jcg :223-232); q1 and rparm1 persist across solves.
__global__ void jcg_clear_lines(unsigned long long *lines, int nwords) {
  griddep_wait();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nwords; k += gridDim.x * blockDim.x)
    lines[k] = kEmpty;
}

__global__ void jcg_init_kernel(Itp *it, Bar *bar, int itmax) {
  griddep_wait();
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
  it->rec.halt = 0;
  it->rec.in = 0;
  it->rec.need_unorm = !it->q1;
}

}  // namespace adc

using namespace adc;

namespace adc {

static size_t round_up(size_t v, size_t m) { return (v + m - 1) / m * m; }

static size_t jcg_stage_bytes(int wmax) { return round_up((size_t)std::max(wmax, 1) * 320, 128); }

// Dynamic shared memory of one block (the largest of the scalar block's
// tridiagonal and a resident row block's layout, see jcg_kernel).
static size_t jcg_smem_bytes(int itmax, bool res, int rows_max, int halo_max, int wmax) {
  size_t tri = round_up(2 * sizeof(double) * (itmax + 1), 128);
  if (!res) return tri;
  size_t rb = (size_t)rows_max, vb = rb + (size_t)halo_max;
  size_t rowb = 8 * rb + 16 * vb + round_up(rb, 128) + 8 * round_up(rb / kSlice, 16) +
                4 * round_up((size_t)halo_max, 32) + 128 + 16 * jcg_stage_bytes(wmax);
  return std::max(tri, rowb);
}

static int jcg_row_block_begin(int nslices, int nrb, int b) {
  return (int)((long long)nslices * b / nrb);
}

// Block-local column indices of the resident variant.  Row block b owns the
// rows of slices [s0, s1); a neighbour in that range maps to its offset
// from the block's first row, any other neighbour to rows_max + its
// position in the block's halo list (first appearance in slot order).
// exp[j] = 1 marks rows that another block reads.
static void jcg_local_tables(int n, int nslices, int nrb, int rows_max, const int *sl_ptr,
                             const int *sl_w, const int *col, const int *rlen,
                             std::vector<unsigned short> &lcol, std::vector<int> &halo_ptr,
                             std::vector<int> &halo_ids, std::vector<unsigned char> &exp,
                             int &halo_max) {
  lcol.assign(std::max(sl_ptr[nslices], 1), 0);
  halo_ptr.assign(nrb + 1, 0);
  halo_ids.clear();
  exp.assign((size_t)nslices * kSlice, 0);
  std::vector<int> stamp(n, -1), hid(n, 0);
  halo_max = 0;
  for (int b = 0; b < nrb; ++b) {
    const int s0 = jcg_row_block_begin(nslices, nrb, b), s1 = jcg_row_block_begin(nslices, nrb, b + 1);
    const int r0 = s0 * kSlice, rows = (s1 - s0) * kSlice;
    int nh = 0;
    for (int sl = s0; sl < s1; ++sl)
      for (int k = 0; k < sl_w[sl]; ++k)
        for (int lane = 0; lane < kSlice; ++lane) {
          const int i = sl * kSlice + lane;
          if (i >= n || k >= rlen[i]) continue;
          const size_t q = (size_t)sl_ptr[sl] + (size_t)k * kSlice + lane;
          const int j = col[q];
          if (j >= r0 && j < r0 + rows) {
            lcol[q] = (unsigned short)(j - r0);
            continue;
          }
          if (stamp[j] != b) {
            stamp[j] = b;
            hid[j] = nh++;
            halo_ids.push_back(j);
            exp[j] = 1;
          }
          lcol[q] = (unsigned short)(rows_max + hid[j]);
        }
    halo_ptr[b + 1] = halo_ptr[b] + nh;
    halo_max = std::max(halo_max, nh);
  }
}

// The dynamic shared memory a kernel may use is a per-function limit that
// every context in the process shares, so it is set to the most the device
// allows (its opt-in maximum less the kernel's static shared memory), not to
// one context's need: contexts with different layouts (the members of an
// ensemble) then all launch.
static int jcg_smem_limit(const void *fn) {
  int dev = 0, optin = 0;
  ADC_CUDA(cudaGetDevice(&dev));
  ADC_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  ADC_CUDA(cudaFuncGetAttributes(&fa, fn));
  ADC_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                optin - (int)fa.sharedSizeBytes));
  return ADC_OK;
}

// Grid of the persistent solver: as many 256-thread row blocks as can be
// co-resident (2 per SM), plus the scalar block.  The resident variant is
// used when host copies of the sliced ELL are given and each row block's
// vectors and staging buffers fit in shared memory at 2 blocks per SM;
// its tables are built and uploaded here.
int jcg_setup_grid(adc_ctx *c, const JcgHostSell *h) {
  int dev = 0, nsm = 0;
  ADC_CUDA(cudaGetDevice(&dev));
  ADC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  if (2 * sizeof(double) * (c->itmax + 1) > 48 * 1024) {
    set_error("itmax too large for the JCG scalar block");
    return ADC_ERR_ARG;
  }
  // keep at least ~8 slices per block so the barrier cost stays amortised
  int nrb0 = std::max(1, std::min(2 * nsm - 1, std::max(1, c->nslices / 8)));
  if (c->jcg_nrb_req > 0) nrb0 = std::max(1, std::min({c->jcg_nrb_req, 2 * nsm - 1, c->nslices}));
  c->jcg_res = 0;
  if (h) {
    const int nrb = nrb0;
    const int rows_max = (c->nslices + nrb - 1) / nrb * kSlice;
    int wmax = 1;
    for (int sl = 0; sl < c->nslices; ++sl) wmax = std::max(wmax, h->sl_w[sl]);
    std::vector<unsigned short> lcol;
    std::vector<int> hptr, hids;
    std::vector<unsigned char> exp;
    int halo_max = 0;
    bool fits = wmax < 128;
    if (fits) {
      jcg_local_tables(c->np, c->nslices, nrb, rows_max, h->sl_ptr, h->sl_w, h->col, h->rlen,
                       lcol, hptr, hids, exp, halo_max);
      fits = rows_max + halo_max < 65536;
    }
    // Stage slices up to width wcap in shared memory; a few wider slices
    // (rows with the most neighbours) are read in place, so that two row
    // blocks still fit on an SM.
    size_t smem = 0;
    int per_sm = 0, wcap = wmax;
    const void *fn = f32_spmv(c) ? (const void *)jcg_kernel<1, float>
                                 : (const void *)jcg_kernel<1, double>;
    for (; fits && wcap >= std::max(1, wmax - 4); --wcap) {
      smem = jcg_smem_bytes(c->itmax, true, rows_max, halo_max, wcap);
      if (smem > 200 * 1024) continue;
      if (int rc = jcg_smem_limit(fn)) return rc;
      ADC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, smem));
      if (per_sm >= 2) break;
    }
    if (per_sm >= 2 && (long long)per_sm * nsm >= nrb + 1) {
      ADC_CUDA(cudaMalloc((void **)&c->jlcol, lcol.size() * sizeof(unsigned short)));
      ADC_CUDA(cudaMemcpy(c->jlcol, lcol.data(), lcol.size() * sizeof(unsigned short),
                          cudaMemcpyHostToDevice));
      ADC_CUDA(cudaMalloc((void **)&c->jhalo_ptr, hptr.size() * sizeof(int)));
      ADC_CUDA(cudaMemcpy(c->jhalo_ptr, hptr.data(), hptr.size() * sizeof(int), cudaMemcpyHostToDevice));
      ADC_CUDA(cudaMalloc((void **)&c->jhalo_ids, std::max<size_t>(hids.size(), 1) * sizeof(int)));
      if (!hids.empty())
        ADC_CUDA(cudaMemcpy(c->jhalo_ids, hids.data(), hids.size() * sizeof(int), cudaMemcpyHostToDevice));
      ADC_CUDA(cudaMalloc((void **)&c->jexp, exp.size()));
      ADC_CUDA(cudaMemcpy(c->jexp, exp.data(), exp.size(), cudaMemcpyHostToDevice));
      c->jcg_rows_blocks = nrb;
      c->jcg_grid = nrb + 1;
      c->jcg_res = 1;
      c->jcg_rows_max = rows_max;
      c->jcg_halo_max = halo_max;
      c->jcg_stage_bytes = (int)jcg_stage_bytes(wcap);
      c->jcg_stage_wcap = wcap;
      c->jcg_smem = smem;
      return ADC_OK;
    }
  }
  const void *fn = (const void *)jcg_kernel<0, double>;
  size_t smem = jcg_smem_bytes(c->itmax, false, 0, 0, 1);
  if (int rc = jcg_smem_limit(fn)) return rc;
  int per_sm = 0;
  ADC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, smem));
  if (per_sm < 1) {
    set_error("jcg kernel cannot be resident");
    return ADC_ERR_CUDA;
  }
  const long long maxb = (long long)per_sm * nsm;
  const int nrb = (int)std::max<long long>(1, std::min<long long>(nrb0, maxb - 1));
  c->jcg_rows_blocks = nrb;
  c->jcg_grid = nrb + 1;
  c->jcg_smem = smem;
  return ADC_OK;
}

int launch_jcg_impl(adc_ctx *c, int eta_update, int do_peror, int run_init, int defer_drift) {
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
  a.soff32 = c->soff32;
  a.diag = c->diag;
  a.rhs = c->gwce_lv;
  a.u = c->etas;
  a.u1 = c->ju1;
  a.p0 = (P4 *)c->jp[0];
  a.p1 = (P4 *)c->jp[1];
  a.w = c->jw;
  a.part = c->jpart;
  a.tri = c->jtri;
  a.itp = c->itp;
  a.bar = c->bar;
  a.arrive = c->jlines;
  a.flags = c->flags;
  a.eta_update = eta_update;
  a.nodecode = c->nodecode;
  a.eta1 = c->eta1;
  a.eta2 = c->eta2;
  a.rows_max = c->jcg_rows_max;
  a.halo_max = c->jcg_halo_max;
  a.stage_bytes = c->jcg_stage_bytes;
  a.stage_wcap = c->jcg_stage_wcap;
  a.lcol = c->jlcol;
  a.halo_ptr = c->jhalo_ptr;
  a.halo_ids = c->jhalo_ids;
  a.exp = c->jexp;
  a.defer_drift = defer_drift;
  // the word after the step flags (allocated only by the time-step context)
  a.drift_pending = defer_drift ? (int *)(c->flags + 1) + 1 : nullptr;
  int nwords = (int)(2 * 128 * (size_t)c->jcg_rows_blocks / 8);
  launch_k(jcg_clear_lines, 8, 256, c->stream, (unsigned long long *)c->jlines, nwords);
  c->launches++;
  if (run_init) {
    launch_k(jcg_init_kernel, 1, 1, c->stream, c->itp, c->bar, c->itmax);
    c->launches++;
  }
  void *args[] = {&a};
  // the FP32 matrix copy exists only for the resident variant of the mixed mode
  const bool vt32 = c->jcg_res && f32_spmv(c) && c->soff32;
  const void *fn = !c->jcg_res ? (const void *)jcg_kernel<0, double>
                   : vt32      ? (const void *)jcg_kernel<1, float>
                               : (const void *)jcg_kernel<1, double>;
  ADC_CUDA(cudaLaunchCooperativeKernel(fn, dim3(c->jcg_grid), dim3(kThreads), args, c->jcg_smem,
                                       c->stream));
  c->launches++;
  return ADC_OK;
}

// The time-step solve defers the COEF drift to the next GWCE (k_lhs_drift).
int launch_jcg(adc_ctx *c, int eta_update) {
  // a mode with FP32 parts keeps no bitwise COEF history, so the drift is dropped
  return launch_jcg_impl(c, eta_update, 0, 1, any_f32(c) ? 2 : 1);
}

}  // namespace adc
