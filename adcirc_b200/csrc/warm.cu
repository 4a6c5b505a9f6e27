// warm.cu -- extrapolated initial guess for the GWCE solve (ADC_WARM_START).
//
// The reference starts JCG from ETAS as GWCE_New leaves it: the previous
// step's increment eta^k - eta^(k-1) at interior nodes and the new boundary
// increment at elevation-specified nodes (gwce.F:1846-1850, 2002-2004).
// With ADC_WARM_START the solve instead starts from the linear
// extrapolation of the increment, 2*ETAS - ETAS_prev, at interior nodes,
// but only when that guess has the smaller initial residual ||b - A u||_2;
// otherwise it keeps the reference guess.  JCG then iterates to the same
// tolerance either way.  The residual norms are fixed-shape FP64 trees, so
// the choice is deterministic.
#include "adc_internal.cuh"

namespace adc {

// Per row: residuals of the reference guess u and of the extrapolated
// guess p = 2u - u_prev (p = u at elevation-specified rows), and their
// block sums of squares.
__global__ void k_warm_resid(adc_ctx c, const double *lg) {
  griddep_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double r2u = 0.0, r2p = 0.0;
  if (i < c.np) {
    const double ui = c.etas[i];
    const double pi = lg ? lg[i] : (c.is_nbd[i] >= 0 ? ui : 2.0 * ui - c.etas_prev[i]);
    const double d = c.diag[i];
    double ru = c.gwce_lv[i] - d * ui;
    double rp = c.gwce_lv[i] - d * pi;
    const int s = i / kSlice, lane = i - s * kSlice;
    const int base = c.sl_ptr[s] + lane, len = c.rlen[i];
    for (int k0 = 0; k0 < len; k0 += kGatherChunk) {
      int jj[kGatherChunk];
      double v[kGatherChunk], uj[kGatherChunk], pj[kGatherChunk];
#pragma unroll
      for (int k = 0; k < kGatherChunk; ++k)
        if (k0 + k < len) {
          const int q = base + (k0 + k) * kSlice;
          jj[k] = c.col[q];
          v[k] = c.offd[q];
        }
#pragma unroll
      for (int k = 0; k < kGatherChunk; ++k)
        if (k0 + k < len) {
          uj[k] = c.etas[jj[k]];
          pj[k] = lg ? lg[jj[k]] : (c.is_nbd[jj[k]] >= 0 ? uj[k] : 2.0 * uj[k] - c.etas_prev[jj[k]]);
        }
#pragma unroll
      for (int k = 0; k < kGatherChunk; ++k)
        if (k0 + k < len) {
          ru = ru - v[k] * uj[k];
          rp = rp - v[k] * pj[k];
        }
    }
    r2u = ru * ru;
    r2p = rp * rp;
  }
  __shared__ double sh[2][32];
  r2u = warp_sum(r2u);
  r2p = warp_sum(r2p);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    sh[0][w] = r2u;
    sh[1][w] = r2p;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    r2u = warp_sum(lane < nw ? sh[0][lane] : 0.0);
    r2p = warp_sum(lane < nw ? sh[1][lane] : 0.0);
    if (lane == 0) {
      c.red[2 * blockIdx.x] = r2u;
      c.red[2 * blockIdx.x + 1] = r2p;
    }
  }
}

// One block: totals in block order, then the choice and its statistics.
__global__ void k_warm_choose(adc_ctx c, int nparts) {
  griddep_wait();
  __shared__ double sh[2][32];
  double su = 0.0, sp = 0.0;
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
    su += c.red[2 * b];
    sp += c.red[2 * b + 1];
  }
  su = warp_sum(su);
  sp = warp_sum(sp);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    sh[0][w] = su;
    sh[1][w] = sp;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    su = warp_sum(lane < nw ? sh[0][lane] : 0.0);
    sp = warp_sum(lane < nw ? sh[1][lane] : 0.0);
    if (lane == 0) {
      const int use = sp < su ? 1 : 0;
      c.warm->use = use;
      if (use) c.warm->n_used++;
      else c.warm->n_fallback++;
    }
  }
}

// Applies the choice.  The extrapolated guess also remembers this step's
// reference guess (the last solution) for the next extrapolation; the
// learned guess `lg` holds the reference guess wherever it predicts
// nothing.
__global__ void k_warm_apply(adc_ctx c, const double *lg) {
  griddep_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.np) return;
  if (lg) {
    if (c.warm->use) c.etas[i] = lg[i];
    return;
  }
  const double u = c.etas[i], uprev = c.etas_prev[i];
  c.etas_prev[i] = u;
  if (c.warm->use && c.is_nbd[i] < 0) c.etas[i] = 2.0 * u - uprev;
}

int launch_predictor_forward(adc_ctx *c);
const double *mp_guess(const adc_ctx *c);

int launch_warm_start(adc_ctx *c) {
  int rc = launch_predictor_forward(c);   // nothing unless a predictor is used or trained
  if (rc) return rc;
  const double *lg = mp_guess(c);
  if (!lg && !(c->prec & ADC_WARM_START)) return ADC_OK;
  const int nb = nblk(c->np);
  launch_k(k_warm_resid, nb, kThreads, c->stream, *c, lg);
  launch_k(k_warm_choose, 1, 1024, c->stream, *c, nb);
  launch_k(k_warm_apply, nb, kThreads, c->stream, *c, lg);
  c->launches += 3;
  return ADC_OK;
}

}  // namespace adc

using namespace adc;

extern "C" int adc_warm_start_stats(adc_ctx *c, long long *used, long long *fallback) {
  if (!c) return ADC_ERR_ARG;
  if (!c->warm) {
    if (used) *used = 0;
    if (fallback) *fallback = 0;
    return ADC_OK;
  }
  WarmState w;
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  ADC_CUDA(cudaMemcpy(&w, c->warm, sizeof(w), cudaMemcpyDeviceToHost));
  if (used) *used = w.n_used;
  if (fallback) *fallback = w.n_fallback;
  return ADC_OK;
}
