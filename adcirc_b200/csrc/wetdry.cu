// wetdry.cu -- computeWettingAndDrying (wetdry.F:140-1470) and computeAlpha
// (wetdry.F:1561-1652): non-subgrid 2DDI, NDDT = 0, default NOFF rules.
// With internal barriers the nodes that receive overflow (NIBNODECODE, set
// by the flux step) wet their elements' nodes through NIBCNT (W2a/W2b,
// wetdry.F:813-816, 1086-1090) and exempt those elements from DE1 (:1114).
//
// Flags are integers and every pass except one is order independent, so
// node and element passes run one thread per item.  The exception is the
// W1 friction update (wetdry.F:593-618): it applies, in element order,
// TK(a) = TK(b) = max(candidate, TK(a), TK(b)) for each wetting event.
// Events are compacted per block in element order, and one block resolves
// the ordered list through each event's predecessors on its two nodes
// (k_wd_chain), which reproduces the sequential result exactly.
#include "adc_internal.cuh"

#include <cfloat>

namespace adc {

constexpr int kW1Block = 256;
constexpr int kChainFast = 1024;   // W1 events resolved in shared memory at a time

// D1, wetdry.F:234-285.
__global__ void k_wd_d1(adc_ctx c) {
  griddep_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) c.flags->n_w1_events = 0;
  if (i >= c.np) return;
  if (c.nodecode[i] == 1) {
    double htot = c.dp[i] + c.eta2[i];
    if (htot <= c.p.h0) {
      double habsmin = 0.8 * c.p.h0;
      if (htot < habsmin) c.eta2[i] = habsmin - c.dp[i];
      c.nnodecode[i] = 0;
      c.nodecode[i] = 0;
      atomicAdd(&c.flags->ncchange, 1);
    }
  }
}

__device__ __forceinline__ double hyb_term(const adc_params_t &p, double h1) {
  if (p.ifhybf == 0) return 0.0;
  return p.ifhybf * pow(1.0 + pow(p.hbreak / h1, p.ftheta), p.fgamma / p.ftheta);
}

// W1, wetdry.F:332-809, plus NOFFOLD/NOFF initialisation (:222-225).
__global__ void __launch_bounds__(kW1Block) k_wd_w1(adc_ctx c) {
  griddep_wait();
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  bool ev = false;
  int ea = 0, eb = 0;
  double ec = 0.0;
  if (e < c.ne) {
    c.noffold[e] = c.noff[e];
    c.noff[e] = 1;
    int NM1 = c.nm[3 * e], NM2 = c.nm[3 * e + 1], NM3 = c.nm[3 * e + 2];
    int nc1 = c.nodecode[NM1], nc2 = c.nodecode[NM2], nc3 = c.nodecode[NM3];
    if (nc1 + nc2 + nc3 == 2) {
      const adc_params_t &p = c.p;
      const double HOFF = 1.2 * p.h0;
      double HT1 = c.dp[NM1] + c.eta2[NM1];
      double HT2 = c.dp[NM2] + c.eta2[NM2];
      double HT3 = c.dp[NM3] + c.eta2[NM3];
      int wa = -1, wb = 0, dry = 0;
      double ha = 0, hb = 0;
      if (nc1 == 1 && nc2 == 1) { wa = NM1; wb = NM2; dry = NM3; ha = HT1; hb = HT2; }
      else if (nc2 == 1 && nc3 == 1) { wa = NM2; wb = NM3; dry = NM1; ha = HT2; hb = HT3; }
      else if (nc3 == 1 && nc1 == 1) { wa = NM3; wb = NM1; dry = NM2; ha = HT3; hb = HT1; }
      if (wa >= 0 && ha >= HOFF && hb >= HOFF) {
        int nm123 = wa;
        if (c.eta2[wb] > c.eta2[wa]) nm123 = wb;
        double dy = c.y[dry] - c.y[nm123], dx = c.x[dry] - c.x[nm123];
        double deldist = sqrt(dy * dy + dx * dx);
        double deleta = c.eta2[nm123] - c.eta2[dry];
        if (deleta < 0.0) deleta = 0.0;
        double h1 = c.eta2[nm123] + c.dp[nm123];
        double fr = c.fric[nm123];
        double tkw = fr * (p.iflinbf + (p.velmin / h1) * (p.ifnlbf + hyb_term(p, h1)));
        double tkwet = (tkw < 0.0001) ? 0.0001 : tkw;   // MAX(., 0.0001)
        double vel = p.g * (deleta / deldist) / tkwet;
        if (vel > p.velmin) {
          c.nnodecode[dry] = 1;
          double tv = fr * (p.iflinbf + (1.0 * vel / h1) * (p.ifnlbf + hyb_term(p, h1)));
          double cap = 2.0 / p.dt;
          ec = (tv < cap) ? tv : cap;
          ea = nm123;
          eb = (nm123 == wa) ? wb : wa;
          ev = true;
        }
      }
    }
  }
  // block-local ordered compaction of the events
  __shared__ int wcnt[kW1Block / 32];
  unsigned m = __ballot_sync(0xffffffffu, ev);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wcnt[w] = __popc(m);
  __syncthreads();
  int off = 0, tot = 0;
  for (int k = 0; k < kW1Block / 32; ++k) {
    if (k < w) off += wcnt[k];
    tot += wcnt[k];
  }
  // each event goes to its block's ordered slot and, while the step has at
  // most kChainFast events, to an unordered list tagged with its element
  __shared__ int s_ubase;
  if (threadIdx.x == 0) {
    c.ev_cnt[blockIdx.x] = tot;
    s_ubase = tot ? atomicAdd(&c.flags->n_w1_events, tot) : 0;
  }
  __syncthreads();
  if (ev) {
    const int r = off + __popc(m & ((1u << lane) - 1u));
    const int pos = blockIdx.x * kW1Block + r;
    c.ev_a[pos] = ea;
    c.ev_b[pos] = eb;
    c.ev_c[pos] = ec;
    const int u = s_ubase + r;
    if (u < kChainFast) {
      c.evu_i[3 * u] = ea;
      c.evu_i[3 * u + 1] = eb;
      c.evu_i[3 * u + 2] = e;
      c.evu_c[u] = ec;
    }
  }
}

// The ordered event list is resolved by the whole block, kChainFast events
// at a time.
// With the events in element order, the value event e assigns is
//   val(e) = max(cand(e), prior(a_e), prior(b_e)),
// where prior(x) is val of the latest earlier event touching node x, or
// the TK that x had before the pass.  Each event's two predecessors are
// found by a backward search; the values then follow by repeated
// max-propagation along those edges until nothing changes (at most the
// depth of the event DAG, each edge pointing to an earlier event), and the
// last event touching a node writes it.  Max is exact, so this equals the
// sequential result bit for bit.

struct ChainSmem {
  int a[kChainFast], b[kChainFast];   // the event's two nodes
  double v[kChainFast];               // candidate, then the value it assigns
  short pa[kChainFast], pb[kChainFast];
  unsigned char lasta[kChainFast], lastb[kChainFast];
  int ord[kChainFast];                // the event's element (its order)
  unsigned long long key[2 * kChainFast];   // (node, order, slot, side) sort keys
};

// k_wd_chain's working set (file scope, so its accesses compile to
// shared-memory instructions).
__shared__ ChainSmem g_chain;

// One chunk of the ordered list.  With `loaded` the chunk's nodes and
// candidates are already in shared memory, else they come from la/lb/lc.
__device__ void chain_block(adc_ctx &c, const int *la, const int *lb, const double *lc,
                            int total, bool loaded) {
  int *s_a = g_chain.a, *s_b = g_chain.b;
  double *s_v = g_chain.v;
  short *s_pa = g_chain.pa, *s_pb = g_chain.pb;
  unsigned char *s_lasta = g_chain.lasta, *s_lastb = g_chain.lastb;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    if (!loaded) {
      s_a[e] = la[e];
      s_b[e] = lb[e];
      s_v[e] = lc[e];   // the event's candidate
      g_chain.ord[e] = e;
    }
    s_lasta[e] = 1;
    s_lastb[e] = 1;
  }
  __syncthreads();
  // predecessors: sort the (node, event, side) pairs; the entry before a
  // pair in sorted order, if it has the same node, is the latest earlier
  // event on that node (bitonic sort in shared memory)
  unsigned long long *key = g_chain.key;
  const int nk = 2 * total;
  int P = 1;
  while (P < nk) P <<= 1;
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    unsigned long long k = ~0ull;   // padding sorts last
    if (i < nk) {
      const int e = i >> 1, side = i & 1;
      const unsigned long long node = (unsigned)(side ? s_b[e] : s_a[e]);
      k = (node << 33) | ((unsigned long long)(unsigned)g_chain.ord[e] << 12) |
          ((unsigned long long)e << 1) | (unsigned long long)side;
    }
    key[i] = k;
  }
  __syncthreads();
  // thread i holds key i (P <= 2 * kChainFast <= 2 * blockDim.x: two keys
  // per thread at most); partners within a warp trade by shuffle, others
  // through shared memory
  for (int kk = 2; kk <= P; kk <<= 1)
    for (int j = kk >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
        for (int i = threadIdx.x; i < P; i += blockDim.x) {
          const int ixj = i ^ j;
          if (ixj > i) {
            const unsigned long long x = key[i], y = key[ixj];
            const bool up = (i & kk) == 0;
            if ((x > y) == up) {
              key[i] = y;
              key[ixj] = x;
            }
          }
        }
        __syncthreads();
      } else {
        // runs of intra-warp stages: every thread updates its own keys
        for (int i0 = threadIdx.x & ~31; i0 < P; i0 += blockDim.x) {
          const int i = i0 + (threadIdx.x & 31);
          unsigned long long x = key[i];
          for (int jj = j; jj > 0; jj >>= 1) {
            const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, jj);
            const bool up = (i & kk) == 0, lower = (i & jj) == 0;
            // the lower partner keeps the min when sorting up, the max otherwise
            const bool keep_min = (lower == up);
            x = keep_min ? (x < y ? x : y) : (x > y ? x : y);
          }
          key[i] = x;
        }
        __syncthreads();
        break;   // the intra-warp stages of this kk are done
      }
    }
  for (int i = threadIdx.x; i < nk; i += blockDim.x) {
    const unsigned long long k = key[i];
    const int e = (int)((k >> 1) & 2047), side = (int)(k & 1);
    int pred = -1;
    if (i > 0 && (key[i - 1] >> 33) == (k >> 33)) pred = (int)((key[i - 1] >> 1) & 2047);
    if (side) s_pb[e] = (short)pred;
    else s_pa[e] = (short)pred;
  }
  __syncthreads();
  // initial values, one thread per event so the global loads overlap
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    double v = s_v[e];
    if (s_pa[e] < 0) {
      const double t = c.tk[s_a[e]];
      if (t > v) v = t;
    }
    if (s_pb[e] < 0) {
      const double t = c.tk[s_b[e]];
      if (t > v) v = t;
    }
    s_v[e] = v;
  }
  __syncthreads();
  // a predecessor found for node x is no longer the last event touching x;
  // each (predecessor, node) pair has one such later event at most
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int pa = s_pa[e], pb = s_pb[e];
    if (pa >= 0) {
      if (s_a[pa] == s_a[e]) s_lasta[pa] = 0;
      else s_lastb[pa] = 0;
    }
    if (pb >= 0) {
      if (s_a[pb] == s_b[e]) s_lasta[pb] = 0;
      else s_lastb[pb] = 0;
    }
  }
  // max-propagation along the predecessor edges (values only grow; a round
  // in which nothing changes is the fixed point); bounded by the list length
  for (int round = 0; round <= total; ++round) {
    int changed = 0;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int pa = s_pa[e], pb = s_pb[e];
      double v = s_v[e];
      double nv = v;
      if (pa >= 0 && s_v[pa] > nv) nv = s_v[pa];
      if (pb >= 0 && s_v[pb] > nv) nv = s_v[pb];
      if (nv != v) {
        s_v[e] = nv;
        changed = 1;
      }
    }
    if (!__syncthreads_or(changed)) break;
  }
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const double v = s_v[e];
    if (s_lasta[e]) {
      const int a = s_a[e];
      c.tk[a] = v;
      c.tkm[3 * a] = v;
      c.tkm[3 * a + 1] = v;
    }
    if (s_lastb[e]) {
      const int b = s_b[e];
      c.tk[b] = v;
      c.tkm[3 * b] = v;
      c.tkm[3 * b + 1] = v;
    }
  }
}

// Sequential-semantics resolution of the W1 TK events (one block).
__global__ void __launch_bounds__(1024) k_wd_chain(adc_ctx c) {
  griddep_wait();
  __shared__ int s_any;
  if (threadIdx.x == 0) s_any = c.flags->n_w1_events;
  __syncthreads();
  if (s_any == 0) return;
  if (s_any <= kChainFast && c.ne < (1 << 21)) {
    // the unordered list W1 wrote: its element tags give the order
    const int total = s_any;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      g_chain.a[e] = c.evu_i[3 * e];
      g_chain.b[e] = c.evu_i[3 * e + 1];
      g_chain.ord[e] = c.evu_i[3 * e + 2];
      g_chain.v[e] = c.evu_c[e];
    }
    __syncthreads();
    chain_block(c, nullptr, nullptr, nullptr, total, true);
    return;
  }
  // long lists: ordered by an exclusive scan of the per-block counts (fixed
  // partition per thread), then resolved in chunks
  const int nb = c.ev_blocks;
  const int T = blockDim.x;
  const int per = (nb + T - 1) / T;
  const int b0 = threadIdx.x * per, b1 = min(nb, b0 + per);
  int mysum = 0;
  for (int b = b0; b < b1; ++b) mysum += c.ev_cnt[b];
  int *sc = (int *)g_chain.key;   // scan scratch, free until the chunks start
  sc[threadIdx.x] = mysum;
  __syncthreads();
  for (int o = 1; o < T; o <<= 1) {
    int v = (threadIdx.x >= (unsigned)o) ? sc[threadIdx.x - o] : 0;
    __syncthreads();
    sc[threadIdx.x] += v;
    __syncthreads();
  }
  const int base = sc[threadIdx.x] - mysum;
  const int total = sc[T - 1];
  // exclusive event offsets of every W1 block (off[nb] = total), then the
  // blocks' events copied into one ordered list by whole warps at a time
  int *off = c.ev_cnt + nb + 1;
  {
    int o = base;
    for (int b = b0; b < b1; ++b) {
      off[b] = o;
      o += c.ev_cnt[b];
    }
    if (threadIdx.x == 0) off[nb] = total;
  }
  __syncthreads();
  int *la = (int *)c.ebuf2;      // ebuf2 holds 3*NE doubles: 2*NE ints, then NE doubles
  int *lb = la + c.ne;
  double *lc = c.ebuf2 + c.ne;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = T >> 5;
  constexpr int kGroup = 8;   // chunks of 32 blocks whose offsets load together
  for (int g0 = warp * 32; g0 < nb; g0 += kGroup * nwarps * 32) {
    int og[kGroup], ng[kGroup];
#pragma unroll
    for (int q = 0; q < kGroup; ++q) {
      const int b = g0 + q * nwarps * 32 + lane;
      og[q] = 0;
      ng[q] = 0;
      if (b < nb) {
        og[q] = off[b];
        ng[q] = off[b + 1] - og[q];
      }
    }
#pragma unroll
    for (int q = 0; q < kGroup; ++q) {
      const int bw = g0 + q * nwarps * 32;
      const int o0 = og[q], n = ng[q];
      unsigned m = __ballot_sync(0xffffffffu, n > 0);
      while (m) {
        const int j = __ffs(m) - 1;
        m &= m - 1;
        const int jo = __shfl_sync(0xffffffffu, o0, j), jn = __shfl_sync(0xffffffffu, n, j);
        for (int k = lane; k < jn; k += 32) {
          const int src = (bw + j) * kW1Block + k, p = jo + k;
          const int ea = c.ev_a[src], eb = c.ev_b[src];
          const double ec = c.ev_c[src];
          if (p < kChainFast) {   // the first chunk goes straight to shared memory
            g_chain.a[p] = ea;
            g_chain.b[p] = eb;
            g_chain.v[p] = ec;
            g_chain.ord[p] = p;
          } else {
            la[p] = ea;
            lb[p] = eb;
            lc[p] = ec;
          }
        }
      }
    }
  }
  __syncthreads();
  // consecutive chunks of the ordered list; a chunk's first events read the
  // TK the previous chunk left in memory
  for (int s0 = 0; s0 < total; s0 += kChainFast) {
    chain_block(c, la + s0, lb + s0, lc + s0, min(kChainFast, total - s0), s0 == 0);
    __syncthreads();
  }
}

// W2a/W2b with internal barriers: NIBCNT(i) sums NIBNODECODE over the nodes
// of every element around node i (wetdry.F:813-816, an integer sum, so its
// element order does not matter), and a node with NIBCNT > 0 is wet
// (:1086-1090).
__global__ void k_wd_w2b(adc_ctx c) {
  griddep_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.np) return;
  int cnt = 0;
  for (int q = c.n2e_ptr[i]; q < c.n2e_ptr[i + 1]; ++q) {
    const int e = c.n2e[q] / 3;
    cnt += c.nib[c.nm[3 * e]] + c.nib[c.nm[3 * e + 1]] + c.nib[c.nm[3 * e + 2]];
  }
  c.nibcnt[i] = cnt;
  if (cnt > 0 && c.nnodecode[i] == 0) c.nnodecode[i] = 1;
}

// DE1 (wetdry.F:1110-1162), then NCEle for D2 and the NOFF change count
// (:1428-1430).
__global__ void k_wd_de1(adc_ctx c) {
  griddep_wait();
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= c.ne) return;
  int NM1 = c.nm[3 * e], NM2 = c.nm[3 * e + 1], NM3 = c.nm[3 * e + 2];
  const double HOFF = 1.2 * c.p.h0;
  double E1 = c.eta2[NM1], E2 = c.eta2[NM2], E3 = c.eta2[NM3];
  double H1 = c.dp[NM1] + E1, H2 = c.dp[NM2] + E2, H3 = c.dp[NM3] + E3;
  int noff = c.noff[e];
  // elements with a barrier-receiving node at every vertex keep NOFF (:1114)
  const bool receiving = c.nfluxib && c.nibcnt[NM1] * c.nibcnt[NM2] * c.nibcnt[NM3] != 0;
  if (!receiving) {
    if ((E1 >= E2) && (E2 > E3)) if ((H1 < HOFF) || (H2 < HOFF)) noff = 0;
    if ((E2 >= E3) && (E3 > E1)) if ((H2 < HOFF) || (H3 < HOFF)) noff = 0;
    if ((E3 >= E1) && (E1 > E2)) if ((H3 < HOFF) || (H1 < HOFF)) noff = 0;
    if ((E1 >= E3) && (E3 > E2)) if ((H1 < HOFF) || (H3 < HOFF)) noff = 0;
    if ((E2 >= E1) && (E1 > E3)) if ((H2 < HOFF) || (H1 < HOFF)) noff = 0;
    if ((E3 >= E2) && (E2 > E1)) if ((H3 < HOFF) || (H2 < HOFF)) noff = 0;
  }
  c.noff[e] = noff;
  c.ncele[e] = c.nnodecode[NM1] * c.nnodecode[NM2] * c.nnodecode[NM3] * noff;
  if (noff != c.noffold[e]) atomicAdd(&c.flags->ncchange, 1);
}

// D2 (wetdry.F:1361-1391), NODECODE update (:1413-1418) and the H2 update
// of timestep.F:1097-1099.
__global__ void k_wd_d2(adc_ctx c) {
  griddep_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.np) return;
  int mju = 0;
  double ta = 0.0;
  const int q0 = c.n2e_ptr[i], q1 = c.n2e_ptr[i + 1];
  for (int qc = q0; qc < q1; qc += kGatherChunk) {
    int ee[kGatherChunk], nc[kGatherChunk];
    double ar[kGatherChunk];
#pragma unroll
    for (int k = 0; k < kGatherChunk; ++k) if (qc + k < q1) ee[k] = c.n2e[qc + k] / 3;
#pragma unroll
    for (int k = 0; k < kGatherChunk; ++k)
      if (qc + k < q1) {
        nc[k] = c.ncele[ee[k]];
        ar[k] = c.areas[ee[k]];
      }
#pragma unroll
    for (int k = 0; k < kGatherChunk; ++k)
      if (qc + k < q1) {
        mju += nc[k];
        ta = ta + nc[k] * ar[k] / 2.0;
      }
  }
  c.totalarea[i] = ta;
  int nn = c.nnodecode[i];
  if (nn == 1 && mju == 0) {
    nn = 0;
    c.nnodecode[i] = 0;
  }
  c.mju[i] = (mju == 0) ? 1 : mju;
  if (nn != c.nodecode[i]) {
    c.nodecode[i] = nn;
    atomicAdd(&c.flags->ncchange, 1);
  }
  c.h2[i] = c.dp[i] + c.p.ifnlfa * c.eta2[i];
}

__global__ void k_h2_update(adc_ctx c) {
  griddep_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.np) return;
  c.h2[i] = c.dp[i] + c.p.ifnlfa * c.eta2[i];
}

// computeAlpha, wetdry.F:1561-1652.
__global__ void k_wd_alpha(adc_ctx c) {
  griddep_wait();
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= c.ne) return;
  int NM1 = c.nm[3 * e], NM2 = c.nm[3 * e + 1], NM3 = c.nm[3 * e + 2];
  double al = 1.0;
  int NCEle = c.nodecode[NM1] * c.nodecode[NM2] * c.nodecode[NM3] * c.noff[e];
  if (NCEle == 1) {
    double E1 = c.eta2[NM1], E2 = c.eta2[NM2], E3 = c.eta2[NM3];
    double HN1 = E1 + c.dp[NM1], HN2 = E2 + c.dp[NM2], HN3 = E3 + c.dp[NM3];
    if ((HN1 <= 5.0e-1) || (HN2 <= 5.0e-1) || (HN3 <= 5.0e-1)) {
      double FDX1 = c.fdx[3 * e], FDX2 = c.fdx[3 * e + 1], FDX3 = c.fdx[3 * e + 2];
      double FDY1 = c.fdy[3 * e], FDY2 = c.fdy[3 * e + 1], FDY3 = c.fdy[3 * e + 2];
      double D1 = c.dp[NM1], D2 = c.dp[NM2], D3 = c.dp[NM3];
      double DPDXA = D1 * FDX1 + D2 * FDX2 + D3 * FDX3;
      double DPDYA = D1 * FDY1 + D2 * FDY2 + D3 * FDY3;
      double DETADXA = E1 * FDX1 + E2 * FDX2 + E3 * FDX3;
      double DETADYA = E1 * FDY1 + E2 * FDY2 + E3 * FDY3;
      double ar = c.areas[e];
      double DPM = sqrt(DPDXA * DPDXA + DPDYA * DPDYA) / ar;
      if (DPM > 1.0e-5) {
        double DDTMP = DETADXA * (-DPDXA) + DETADYA * (-DPDYA);
        if (fabs(DDTMP) > 1.0e-12)
          al = c.p.slim * (sqrt(DPDXA * DPDXA + DPDYA * DPDYA) / ((1.0 / ar) * (DDTMP)));
        else
          al = 1.0;
      } else {
        double DETAM = sqrt(DETADXA * DETADXA + DETADYA * DETADYA) / ar;
        if (fabs(DETAM) > 1.0e-12) al = c.p.slim / DETAM;
        else al = 1.0;
      }
      if (al <= 0.0) al = 1.0;
      if (al >= 1.0) al = 1.0;
    }
  }
  c.alphal[e] = al;
}

int launch_wetdry(adc_ctx *c) {
  const adc_ctx &cv = *c;
  if (c->p.nolifa != 2) {
    launch_k(k_h2_update, nblk(c->np), kThreads, c->stream, cv);
    c->launches++;
    return ADC_OK;
  }
  launch_k(k_wd_d1, nblk(c->np), kThreads, c->stream, cv);
  launch_k(k_wd_w1, c->ev_blocks, kW1Block, c->stream, cv);
  launch_k(k_wd_chain, 1, 1024, c->stream, cv);
  if (c->nfluxib) {
    launch_k(k_wd_w2b, nblk(c->np), kThreads, c->stream, cv);
    c->launches++;
  }
  launch_k(k_wd_de1, nblk(c->ne), kThreads, c->stream, cv);
  launch_k(k_wd_d2, nblk(c->np), kThreads, c->stream, cv);
  launch_k(k_wd_alpha, nblk(c->ne), kThreads, c->stream, cv);
  c->launches += 6;
  return ADC_OK;
}

}  // namespace adc
