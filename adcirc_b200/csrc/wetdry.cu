// wetdry.cu -- computeWettingAndDrying (wetdry.F:140-1470) and computeAlpha
// (wetdry.F:1561-1652): non-subgrid 2DDI, no weirs or barriers
// (NIBNODECODE = 0, so W2a/W2b never fire), NDDT = 0, default NOFF rules.
//
// Flags are integers and every pass except one is order independent, so
// node and element passes run one thread per item.  The exception is the
// W1 friction update (wetdry.F:593-618): it applies, in element order,
// TK(a) = TK(b) = max(candidate, TK(a), TK(b)) for each wetting event.
// Events are compacted per block in element order and resolved by one warp
// in batches of 32, with in-batch dependencies settled by shuffles, which
// reproduces the sequential result exactly.
#include "adc_internal.cuh"

#include <cfloat>

namespace adc {

constexpr int kW1Block = 256;

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
  if (ev) {
    int pos = blockIdx.x * kW1Block + off + __popc(m & ((1u << lane) - 1u));
    c.ev_a[pos] = ea;
    c.ev_b[pos] = eb;
    c.ev_c[pos] = ec;
  }
  if (threadIdx.x == 0) {
    c.ev_cnt[blockIdx.x] = tot;
    if (tot) atomicAdd(&c.flags->n_w1_events, tot);
  }
}

// Sequential-semantics resolution of the W1 TK events (one block).
__global__ void __launch_bounds__(1024) k_wd_chain(adc_ctx c) {
  griddep_wait();
  __shared__ int s_any;
  if (threadIdx.x == 0) s_any = c.flags->n_w1_events;
  __syncthreads();
  if (s_any == 0) return;
  // exclusive scan of the per-block counts (fixed partition per thread)
  const int nb = c.ev_blocks;
  const int T = blockDim.x;
  const int per = (nb + T - 1) / T;
  const int b0 = threadIdx.x * per, b1 = min(nb, b0 + per);
  int mysum = 0;
  for (int b = b0; b < b1; ++b) mysum += c.ev_cnt[b];
  __shared__ int sc[1024];
  sc[threadIdx.x] = mysum;
  __syncthreads();
  for (int o = 1; o < T; o <<= 1) {
    int v = (threadIdx.x >= (unsigned)o) ? sc[threadIdx.x - o] : 0;
    __syncthreads();
    sc[threadIdx.x] += v;
    __syncthreads();
  }
  int base = sc[threadIdx.x] - mysum;
  const int total = sc[T - 1];
  // gather events into one contiguous ordered list (reuses ebuf2 as doubles
  // for candidates and the tail of ev arrays is not touched)
  int *la = (int *)c.ebuf2;
  int *lb = la + c.ne;
  double *lc = c.ebuf2 + c.ne;   // ebuf2 holds 3*NE doubles
  for (int b = b0; b < b1; ++b) {
    int n = c.ev_cnt[b];
    for (int k = 0; k < n; ++k) {
      int src = b * kW1Block + k;
      la[base + k] = c.ev_a[src];
      lb[base + k] = c.ev_b[src];
      lc[base + k] = c.ev_c[src];
    }
    base += n;
  }
  __syncthreads();
  __threadfence_block();
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  for (int s = 0; s < total; s += 32) {
    int m = min(32, total - s);
    bool act = lane < m;
    int a = act ? la[s + lane] : -1 - lane;
    int b = act ? lb[s + lane] : -1000 - lane;
    double cand = act ? lc[s + lane] : 0.0;
    double A = act ? c.tk[a] : 0.0;
    double B = act ? c.tk[b] : 0.0;
    int pa = -1, pb = -1;
    bool last_a = true, last_b = true;
    for (int j = 0; j < 32; ++j) {
      int aj = __shfl_sync(0xffffffffu, a, j);
      int bj = __shfl_sync(0xffffffffu, b, j);
      if (j < lane) {
        if (aj == a || bj == a) pa = j;
        if (aj == b || bj == b) pb = j;
      } else if (j > lane && j < m) {
        if (aj == a || bj == a) last_a = false;
        if (aj == b || bj == b) last_b = false;
      }
    }
    double v = cand;
    if (pa < 0 && A > v) v = A;
    if (pb < 0 && B > v) v = B;
    for (int r = 0; r < 33; ++r) {
      double va = __shfl_sync(0xffffffffu, v, pa >= 0 ? pa : lane);
      double vb = __shfl_sync(0xffffffffu, v, pb >= 0 ? pb : lane);
      double nv = v;
      if (pa >= 0 && va > nv) nv = va;
      if (pb >= 0 && vb > nv) nv = vb;
      bool ch = nv != v;
      v = nv;
      if (!__any_sync(0xffffffffu, ch)) break;
    }
    if (act && last_a) {
      c.tk[a] = v;
      c.tkm[3 * a] = v;
      c.tkm[3 * a + 1] = v;
    }
    if (act && last_b) {
      c.tk[b] = v;
      c.tkm[3 * b] = v;
      c.tkm[3 * b + 1] = v;
    }
    __syncwarp();
  }
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
  if ((E1 >= E2) && (E2 > E3)) if ((H1 < HOFF) || (H2 < HOFF)) noff = 0;
  if ((E2 >= E3) && (E3 > E1)) if ((H2 < HOFF) || (H3 < HOFF)) noff = 0;
  if ((E3 >= E1) && (E1 > E2)) if ((H3 < HOFF) || (H1 < HOFF)) noff = 0;
  if ((E1 >= E3) && (E3 > E2)) if ((H1 < HOFF) || (H3 < HOFF)) noff = 0;
  if ((E2 >= E1) && (E1 > E3)) if ((H2 < HOFF) || (H1 < HOFF)) noff = 0;
  if ((E3 >= E2) && (E2 > E1)) if ((H3 < HOFF) || (H2 < HOFF)) noff = 0;
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
  launch_k(k_wd_de1, nblk(c->ne), kThreads, c->stream, cv);
  launch_k(k_wd_d2, nblk(c->np), kThreads, c->stream, cv);
  launch_k(k_wd_alpha, nblk(c->ne), kThreads, c->stream, cv);
  c->launches += 6;
  return ADC_OK;
}

}  // namespace adc
