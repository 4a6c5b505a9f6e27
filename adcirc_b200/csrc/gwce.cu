// gwce.cu -- GWCE_New (gwce.F:237-2111) for IM=0 (Kolar-Gray lateral
// stress, non-conservative advection), consistent mass (ILump = 0),
// Cartesian coordinates, plus the TIMESTEP glue that precedes it.
//
// Element terms are computed once per element into a scratch buffer and
// gathered per node over the node->element CSR in increasing element order,
// i.e. the order of the reference's scatter loops, starting from zero as
// the reference does after zeroing.  No atomics touch floating point, so
// the results are deterministic and, compiled without FMA contraction,
// reproduce the serial arithmetic bit for bit.
#include "adc_internal.cuh"

namespace adc {

// --------------------------------------------------------------- shift
// timestep.F:231-237 (IT==1 H init), :375-416 (time-level shift, zeroing),
// nodalattr.F:2399-2413 (quadratic/linear/hybrid friction), :2700-2704.
__global__ void k_shift_friction(adc_ctx c, const adc_step_t *steps, const Flags *flags) {
  griddep_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.np) return;
  const adc_step_t st = steps[flags->cursor];
  const adc_params_t &p = c.p;
  if (st.it == 1) {
    double h = c.dp[i] + p.ifnlfa * c.eta2[i];
    c.h2[i] = h;
    c.h1[i] = h;
  }
  c.qx1[i] = c.qx2[i];
  c.qy1[i] = c.qy2[i];
  double u1 = c.uu2[i], v1 = c.vv2[i];
  c.uu1[i] = u1;
  c.vv1[i] = v1;
  c.gwce_lv[i] = 0.0;
  c.mom_x[i] = 0.0;
  c.mom_y[i] = 0.0;
  if (p.nws != 0) {
    c.wsx1[i] = c.wsx2[i];
    c.wsx2[i] = 0.0;
    c.wsy1[i] = c.wsy2[i];
    c.wsy2[i] = 0.0;
    c.pr1[i] = c.pr2[i];
  }
  c.pr2[i] = p.prbckgrnd_mh2o;
  double uv1 = sqrt(u1 * u1 + v1 * v1);
  double h1 = c.dp[i] + p.ifnlfa * c.eta2[i];
  double hyb = 0.0;
  if (p.ifhybf != 0) hyb = p.ifhybf * pow(1.0 + pow(p.hbreak / h1, p.ftheta), p.fgamma / p.ftheta);
  double v = c.fric[i] * (p.iflinbf + (uv1 / h1) * (p.ifnlbf + hyb));
  double cap = 2.0 / p.dt;
  double tk = (v < cap) ? v : cap;
  c.tk[i] = tk;
  c.tkm[3 * i + 0] = tk;
  c.tkm[3 * i + 1] = tk;
  c.tkm[3 * i + 2] = 0.0;
  if (c.nfluxib) c.nib[i] = 0;   // NIBNODECODE(:) = 0, timestep.F:1004
}

// Met forcing supplied by the host for this step (WSX2, WSY2, PR2).
__global__ void k_apply_met(adc_ctx c) {
  griddep_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.np) return;
  c.wsx2[i] = c.met_wsx[i];
  c.wsy2[i] = c.met_wsy[i];
  c.pr2[i] = c.met_pr[i];
}

// --------------------------------------------------------------- LHS
// The rebuild runs only when NCChange > 0 (gwce.F:430-431).  words[0] is
// the rebuild decision; words[1] is set by a solve that left the ITPACK
// unscal drift of COEF pending; words[2] says whether this step applies it
// (only when COEF is kept, since a rebuild overwrites it).
__global__ void k_lhs_begin(Flags *f, int *words) {
  griddep_wait();
  int r = f->ncchange > 0;
  words[0] = r;
  words[2] = (!r && words[1]) ? 1 : 0;
  words[1] = 0;
  if (r) f->ncchange = 0;
}

// Moves the COEF drift from a point after the solve to the next step that
// keeps COEF, so steps that rebuild COEF never pay for it.  It repeats the
// exact operations of the solve's scal/unscal pass (itpackv.F:2393-2398,
// 2458-2463) with the w = 1/sqrt(diag) that solve used, so COEF ends with
// the same bits as if the solve had written it.
__global__ void k_lhs_drift(adc_ctx c, const int *apply) {
  griddep_wait();
  if (!*apply) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  // the drift changes every row's off-diagonals: the next rebuild gathers all
  if (i == 0) const_cast<int *>(apply)[1] = 1;
  if (i >= c.np) return;
  const double wi = c.jw[i];
  const double winv_i = 1.0 / wi;
  const int s = i / kSlice, lane = i - s * kSlice;
  const int base = c.sl_ptr[s] + lane, len = c.rlen[i];
  for (int k = 0; k < len; ++k) {
    const int q = base + k * kSlice;
    const double wj = c.jw[c.col[q]];
    const double sv = c.offd[q] * wi * wj;
    c.offd[q] = sv * winv_i * (1.0 / wj);
  }
}

// Single-thread helper: make a pending drift apply now (before COEF is
// copied to the host).
__global__ void k_lhs_drift_flush(int *words) {
  griddep_wait();
  words[2] = words[1];
  words[1] = 0;
}

// gwce.F:456-593: nine consistent-mass + gravity entries per element.
// The entries depend on the element's static geometry and depth and on two
// per-step inputs, NCEle and ALPHAL; an element is recomputed only when
// those differ from the values its cached entries were built with (every
// element on the first rebuild and after a host upload), and the nodes of
// a recomputed element are marked for the row gather.  The cached entries
// equal what a full rebuild writes, bit for bit.
template <class R>
__global__ void k_lhs_elem(adc_ctx c, const int *rebuild) {
  griddep_wait();
  if (!*rebuild) return;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= c.ne) return;
  int n1 = c.nm[3 * e], n2 = c.nm[3 * e + 1], n3 = c.nm[3 * e + 2];
  int NCEle = c.nodecode[n1] * c.nodecode[n2] * c.nodecode[n3] * c.noff[e];
  const double ald = c.alphal[e];
  if (c.lhs_nc[e] == NCEle &&
      __double_as_longlong(c.lhs_al[e]) == __double_as_longlong(ald))
    return;
  const adc_params_t &p = c.p;
  const R DT = R(p.dt);
  R FDX1 = c.fdx[3 * e], FDX2 = c.fdx[3 * e + 1], FDX3 = c.fdx[3 * e + 2];
  R FDY1 = c.fdy[3 * e], FDY2 = c.fdy[3 * e + 1], FDY3 = c.fdy[3 * e + 2];
  R AreaIE2 = c.areas[e];
  R AreaIE = AreaIE2 * R(0.5);
  R AreaIE4 = AreaIE2 * R(2.0);
  R DPAvg = (c.dp[n1] + c.dp[n2] + c.dp[n3]) / R(3.0);
  R GA = R(ald) * R(p.a00) * R(p.g) * DPAvg / AreaIE4;
  R Tau0Avg = (c.tau0[n1] + c.tau0[n2] + c.tau0[n3]) / R(3.0);
  R MsOn = 2 * AreaIE * (R(1.0) / DT + Tau0Avg / R(2.0)) / DT / R(12.0);
  R MsOff = 1 * AreaIE * (R(1.0) / DT + Tau0Avg / R(2.0)) / DT / R(12.0);
  R nc = (R)NCEle;
  R *o = reinterpret_cast<R *>(c.lhs_ebuf) + 9 * (size_t)e;
  o[0] = (MsOn + GA * (FDX1 * FDX1 + FDY1 * FDY1)) * nc;
  o[1] = (MsOn + GA * (FDX2 * FDX2 + FDY2 * FDY2)) * nc;
  o[2] = (MsOn + GA * (FDX3 * FDX3 + FDY3 * FDY3)) * nc;
  o[3] = (MsOff + GA * (FDX1 * FDX2 + FDY1 * FDY2)) * nc;  // (n1, J12)
  o[4] = (MsOff + GA * (FDX1 * FDX3 + FDY1 * FDY3)) * nc;  // (n1, J13)
  o[5] = (MsOff + GA * (FDX2 * FDX1 + FDY2 * FDY1)) * nc;  // (n2, J21)
  o[6] = (MsOff + GA * (FDX2 * FDX3 + FDY2 * FDY3)) * nc;  // (n2, J23)
  o[7] = (MsOff + GA * (FDX3 * FDX1 + FDY3 * FDY1)) * nc;  // (n3, J31)
  o[8] = (MsOff + GA * (FDX3 * FDX2 + FDY3 * FDY2)) * nc;  // (n3, J32)
  c.lhs_nc[e] = NCEle;
  c.lhs_al[e] = ald;
  c.lhs_dirty[n1] = 1;
  c.lhs_dirty[n2] = 1;
  c.lhs_dirty[n3] = 1;
}

// Per-row gather of COEF in element order, and the per-block partial of
// sum(diag^2) for EP (gwce.F:646-650).
template <class R>
__global__ void k_lhs_gather(adc_ctx c, const int *rebuild) {
  griddep_wait();
  if (!*rebuild) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const R *eb = reinterpret_cast<const R *>(c.lhs_ebuf);
  double d2 = 0.0;
  // rows whose elements did not change keep their gathered off-diagonals;
  // only their diagonal, which each solve's scal/unscal rewrites, returns
  // to the gathered value
  const bool all = rebuild[3] != 0;
  if (i < c.np && !all && !c.lhs_dirty[i] && !c.bc_row[i]) {
    const double d = c.diag_gathered[i];
    c.diag[i] = d;
    d2 = d * d;
  } else if (i < c.np) {
    R d = R(0.0);
    const int q0 = c.n2e_ptr[i], q1 = c.n2e_ptr[i + 1];
    for (int qc = q0; qc < q1; qc += kGatherChunk) {
      int ek[kGatherChunk];
      R x[kGatherChunk];
#pragma unroll
      for (int k = 0; k < kGatherChunk; ++k) if (qc + k < q1) ek[k] = c.n2e[qc + k];
#pragma unroll
      for (int k = 0; k < kGatherChunk; ++k)
        if (qc + k < q1) {
          int e = ek[k] / 3, kk = ek[k] - 3 * e;
          x[k] = eb[9 * (size_t)e + kk];
        }
#pragma unroll
      for (int k = 0; k < kGatherChunk; ++k) if (qc + k < q1) d = d + x[k];
    }
    c.diag[i] = (double)d;
    c.diag_gathered[i] = (double)d;
    c.lhs_dirty[i] = 0;
    d2 = (double)d * (double)d;
    int s = i / kSlice, lane = i - s * kSlice;
    int base = c.sl_ptr[s] + lane;
    int len = c.rlen[i];
    for (int kc = 0; kc < len; kc += kGatherChunk) {
      int2 src[kGatherChunk];
      R va[kGatherChunk], vb[kGatherChunk];
#pragma unroll
      for (int k = 0; k < kGatherChunk; ++k)
        if (kc + k < len) src[k] = reinterpret_cast<const int2 *>(c.lhs_src)[base + (kc + k) * kSlice];
#pragma unroll
      for (int k = 0; k < kGatherChunk; ++k)
        if (kc + k < len) {
          va[k] = src[k].x >= 0 ? eb[src[k].x] : R(0.0);
          vb[k] = src[k].y >= 0 ? eb[src[k].y] : R(0.0);
        }
#pragma unroll
      for (int k = 0; k < kGatherChunk; ++k)
        if (kc + k < len) {
          R v = R(0.0);
          if (src[k].x >= 0) v = v + va[k];
          if (src[k].y >= 0) v = v + vb[k];
          c.offd[base + (kc + k) * kSlice] = (double)v;
        }
    }
  }
  __shared__ double sh[32];
  d2 = warp_sum(d2);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = d2;
  __syncthreads();
  if (w == 0) {
    d2 = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    d2 = warp_sum(d2);
    if (lane == 0) c.red[blockIdx.x] = d2;
  }
}

__global__ void k_lhs_ep(adc_ctx c, const int *rebuild, int nparts) {
  griddep_wait();
  if (!*rebuild) return;
  __shared__ double sh[32];
  double s = 0.0;
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) s += c.red[b];
  s = warp_sum(s);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = s;
  __syncthreads();
  if (w == 0) {
    s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    s = warp_sum(s);
    if (lane == 0) {
      c.flags->ep = sqrt(s / c.np);
      *const_cast<int *>(rebuild + 3) = 0;   // every row is gathered again
    }
  }
}

// gwce.F:654-707: elevation-boundary rows and columns, OBCCoef, diagonal
// checks.  Thread t < NP handles row t; thread NP + q handles the q-th
// (I, J) column entry.
__global__ void k_lhs_bc(adc_ctx c, const int *rebuild) {
  griddep_wait();
  if (!*rebuild) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const double EP = c.flags->ep;
  if (t < c.np) {
    int i = t;
    if (c.is_nbd[i] >= 0) {
      c.diag[i] = EP;
      int s = i / kSlice, lane = i - s * kSlice;
      int base = c.sl_ptr[s] + lane;
      int len = c.rlen[i];
      for (int k = 0; k < len; ++k) c.offd[base + k * kSlice] = 0.0;
    }
    double d = c.diag[i];
    if (d == 0.0) {
      d = EP;
      c.diag[i] = d;
    }
    if (d < 0.0) atomicExch(&c.flags->status, ADC_ERR_DIAG);
    return;
  }
  int q = t - c.np;
  if (q >= c.n_obc) return;
  int slot = c.obc_slot[q];
  double v = 0.0;
  if (slot >= 0) {
    if (!c.obc_zero[q]) v = c.offd[slot];
    c.offd[slot] = 0.0;
  }
  c.obccoef[q] = v;
}

// --------------------------------------------------------------- RHS
// gwce.F:1000-1617, one element, IM=0 branches.
template <class R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 3 : 2) k_rhs_elem(adc_ctx c) {
  griddep_wait();
  __shared__ R sh[kThreads / 32][32 * 3];
  const int e0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31);
  if (e0 >= c.ne) return;
  const int nvalid = min(32, c.ne - e0);
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= c.ne) e = c.ne - 1;   // idle lanes recompute the last element; not stored
  const adc_params_t &p = c.p;
  const R DT = R(p.dt), G = R(p.g), A00 = R(p.a00), B00 = R(p.b00), C00 = R(p.c00);
  // x / DT: with a power-of-two DT, the product with its exact reciprocal
  // gives the same bits
  const bool dt2 = c.dt_pow2 != 0;
  const R IDT = R(c.inv_dt);
  auto odt = [&](R x) { return dt2 ? x * IDT : x / DT; };
  int n1 = c.nm[3 * e], n2 = c.nm[3 * e + 1], n3 = c.nm[3 * e + 2];
  int NCEle = c.nodecode[n1] * c.nodecode[n2] * c.nodecode[n3] * c.noff[e];
  R E0N1 = c.eta1[n1], E0N2 = c.eta1[n2], E0N3 = c.eta1[n3];
  R E1N1 = c.eta2[n1], E1N2 = c.eta2[n2], E1N3 = c.eta2[n3];
  R E1N1SQ = E1N1 * E1N1, E1N2SQ = E1N2 * E1N2, E1N3SQ = E1N3 * E1N3;
  R ESN1 = c.etas[n1], ESN2 = c.etas[n2], ESN3 = c.etas[n3];
  R U1N1 = c.uu1[n1], U1N2 = c.uu1[n2], U1N3 = c.uu1[n3];
  R V1N1 = c.vv1[n1], V1N2 = c.vv1[n2], V1N3 = c.vv1[n3];
  R QX1N1 = c.qx1[n1], QX1N2 = c.qx1[n2], QX1N3 = c.qx1[n3];
  R QY1N1 = c.qy1[n1], QY1N2 = c.qy1[n2], QY1N3 = c.qy1[n3];
  R H1N1 = c.h2[n1], H1N2 = c.h2[n2], H1N3 = c.h2[n3];
  R EVMN1 = c.evm[n1], EVMN2 = c.evm[n2], EVMN3 = c.evm[n3];
  R T0N1 = c.tau0[n1], T0N2 = c.tau0[n2], T0N3 = c.tau0[n3];
  const bool met = p.nws != 0;
  R Pr1N1 = R(0.0), Pr1N2 = R(0.0), Pr1N3 = R(0.0);
  if (met) {
    if constexpr (sizeof(R) == 4) {
      // only the gradient of PR1 is used: FP32 carries its deviation from
      // the background pressure, not the ~10 m total
      const double pb = p.prbckgrnd_mh2o;
      Pr1N1 = R(c.pr1[n1] - pb); Pr1N2 = R(c.pr1[n2] - pb); Pr1N3 = R(c.pr1[n3] - pb);
    } else {
      Pr1N1 = c.pr1[n1]; Pr1N2 = c.pr1[n2]; Pr1N3 = c.pr1[n3];
    }
  }
  const double *tk1 = c.tkm + 3 * n1, *tk2 = c.tkm + 3 * n2, *tk3 = c.tkm + 3 * n3;
  R BSXN1 = R(tk1[0]) * QX1N1 + R(tk1[2]) * QY1N1;
  R BSYN1 = R(tk1[2]) * QX1N1 + R(tk1[1]) * QY1N1;
  R BSXN2 = R(tk2[0]) * QX1N2 + R(tk2[2]) * QY1N2;
  R BSYN2 = R(tk2[2]) * QX1N2 + R(tk2[1]) * QY1N2;
  R BSXN3 = R(tk3[0]) * QX1N3 + R(tk3[2]) * QY1N3;
  R BSYN3 = R(tk3[2]) * QX1N3 + R(tk3[1]) * QY1N3;
  R AreaIE2 = c.areas[e];
  R AreaIE = AreaIE2 / R(2.0);
  R AreaIE4 = R(2.0) * AreaIE2;
  R FDX1 = c.fdx[3 * e], FDX2 = c.fdx[3 * e + 1], FDX3 = c.fdx[3 * e + 2];
  R FDY1 = c.fdy[3 * e], FDY2 = c.fdy[3 * e + 1], FDY3 = c.fdy[3 * e + 2];
  R E0XGrad2A, E0YGrad2A, E1XGrad2A, E1YGrad2A, E1SQXGrad2A, E1SQYGrad2A;
  if constexpr (sizeof(R) == 4) {
    // Elevation gradients cancel metre-sized nodal values down to
    // centimetres: they are formed in FP64 and only then narrowed.
    const double *fx = c.fdx + 3 * e, *fy = c.fdy + 3 * e;
    const double a1 = c.eta1[n1], a2 = c.eta1[n2], a3 = c.eta1[n3];
    const double b1 = c.eta2[n1], b2 = c.eta2[n2], b3 = c.eta2[n3];
    E0XGrad2A = R(a1 * fx[0] + a2 * fx[1] + a3 * fx[2]);
    E0YGrad2A = R(a1 * fy[0] + a2 * fy[1] + a3 * fy[2]);
    E1XGrad2A = R(b1 * fx[0] + b2 * fx[1] + b3 * fx[2]);
    E1YGrad2A = R(b1 * fy[0] + b2 * fy[1] + b3 * fy[2]);
    E1SQXGrad2A = R(b1 * b1 * fx[0] + b2 * b2 * fx[1] + b3 * b3 * fx[2]);
    E1SQYGrad2A = R(b1 * b1 * fy[0] + b2 * b2 * fy[1] + b3 * b3 * fy[2]);
  } else {
    E0XGrad2A = E0N1 * FDX1 + E0N2 * FDX2 + E0N3 * FDX3;
    E0YGrad2A = E0N1 * FDY1 + E0N2 * FDY2 + E0N3 * FDY3;
    E1XGrad2A = E1N1 * FDX1 + E1N2 * FDX2 + E1N3 * FDX3;
    E1YGrad2A = E1N1 * FDY1 + E1N2 * FDY2 + E1N3 * FDY3;
    E1SQXGrad2A = E1N1SQ * FDX1 + E1N2SQ * FDX2 + E1N3SQ * FDX3;
    E1SQYGrad2A = E1N1SQ * FDY1 + E1N2SQ * FDY2 + E1N3SQ * FDY3;
  }
  R Tau0XGrad2A = T0N1 * FDX1 + T0N2 * FDX2 + T0N3 * FDX3;
  R Tau0YGrad2A = T0N1 * FDY1 + T0N2 * FDY2 + T0N3 * FDY3;
  R EVMXGrad = (EVMN1 * FDX1 + EVMN2 * FDX2 + EVMN3 * FDX3) / AreaIE2;
  R EVMYGrad = (EVMN1 * FDY1 + EVMN2 * FDY2 + EVMN3 * FDY3) / AreaIE2;
  R EVMAvgODT = odt(div3(EVMN1 + EVMN2 + EVMN3));
  R MX = (EVMXGrad * (QX1N1 * FDX1 + QX1N2 * FDX2 + QX1N3 * FDX3) +
               EVMYGrad * (QY1N1 * FDX1 + QY1N2 * FDX2 + QY1N3 * FDX3) -
               EVMAvgODT * (ESN1 * FDX1 + ESN2 * FDX2 + ESN3 * FDX3)) / AreaIE2;
  R MY = (EVMXGrad * (QX1N1 * FDY1 + QX1N2 * FDY2 + QX1N3 * FDY3) +
               EVMYGrad * (QY1N1 * FDY1 + QY1N2 * FDY2 + QY1N3 * FDY3) -
               EVMAvgODT * (ESN1 * FDY1 + ESN2 * FDY2 + ESN3 * FDY3)) / AreaIE2;
  R CorifAvg = div3(c.corif[n1] + c.corif[n2] + c.corif[n3]);
  R Tau0Avg = div3(T0N1 + T0N2 + T0N3);
  R Tau0QXAvg = div3(T0N1 * QX1N1 + T0N2 * QX1N2 + T0N3 * QX1N3);
  R Tau0QYAvg = div3(T0N1 * QY1N1 + T0N2 * QY1N2 + T0N3 * QY1N3);
  R U1Avg = div3(U1N1 + U1N2 + U1N3);
  R V1Avg = div3(V1N1 + V1N2 + V1N3);
  R QX1Avg = div3(QX1N1 + QX1N2 + QX1N3);
  R QY1Avg = div3(QY1N1 + QY1N2 + QY1N3);
  R ESAvg = div3(ESN1 + ESN2 + ESN3);
  R DPAvg = div3(c.dp[n1] + c.dp[n2] + c.dp[n3]);
  R al = c.alphal[e];
  R GDPAvgOAreaIE4 = al * G * DPAvg / AreaIE4;
  R GDPAvgOAreaIE4_S0 = GDPAvgOAreaIE4;   // DPAvgS0 == DPAvg when IFNL_HDP = 0
  R HAvg = div3(H1N1 + H1N2 + H1N3);
  R GHAvg = al * G * HAvg;
  R GHAvgOAreaIE2 = GHAvg / AreaIE2;
  R BSXAvg = div3(BSXN1 + BSXN2 + BSXN3);
  R BSYAvg = div3(BSYN1 + BSYN2 + BSYN3);
  R WSXAvg = R(0.0), WSYAvg = R(0.0);
  if (met) {
    WSXAvg = div3(c.wsx1[n1] + c.wsx1[n2] + c.wsx1[n3]);
    WSYAvg = div3(c.wsy1[n1] + c.wsy1[n2] + c.wsy1[n3]);
  }
  R MsFacR = div12(odt(AreaIE * ((dt2 ? IDT : R(1.0) / DT) - Tau0Avg / R(2.0))));
  R GOAreaIE4 = al * G / AreaIE4;
  R Tau0SpaVar = div6(QX1Avg * Tau0XGrad2A + QY1Avg * Tau0YGrad2A);
  R A00pB00 = A00 + B00;
  R fa = p.ifnlfa * GOAreaIE4;
  R JXAvg = CorifAvg * QY1Avg - fa * E1SQXGrad2A -
                 GHAvgOAreaIE2 * (Pr1N1 * FDX1 + Pr1N2 * FDX2 + Pr1N3 * FDX3) + WSXAvg -
                 BSXAvg + MX + Tau0QXAvg;
  R JYAvg = -CorifAvg * QX1Avg - fa * E1SQYGrad2A -
                 GHAvgOAreaIE2 * (Pr1N1 * FDY1 + Pr1N2 * FDY2 + Pr1N3 * FDY3) + WSYAvg -
                 BSYAvg + MY + Tau0QYAvg;
  JXAvg = JXAvg - p.ifnlct * (QX1Avg * (U1N1 * FDX1 + U1N2 * FDX2 + U1N3 * FDX3) +
                              QY1Avg * (U1N1 * FDY1 + U1N2 * FDY2 + U1N3 * FDY3)) / AreaIE2 +
          odt(p.ifnlcat * U1Avg * ESAvg);
  JYAvg = JYAvg - p.ifnlct * (QX1Avg * (V1N1 * FDX1 + V1N2 * FDX2 + V1N3 * FDX3) +
                              QY1Avg * (V1N1 * FDY1 + V1N2 * FDY2 + V1N3 * FDY3)) / AreaIE2 +
          odt(p.ifnlcat * V1Avg * ESAvg);
  R c0 = GDPAvgOAreaIE4_S0, c1 = GDPAvgOAreaIE4;
  R T1 = (2 * ESN1 + 1 * (ESN2 + ESN3)) * MsFacR -
              c0 * (C00 * (FDX1 * E0XGrad2A + FDY1 * E0YGrad2A)) -
              c1 * (A00pB00 * (FDX1 * E1XGrad2A + FDY1 * E1YGrad2A)) +
              (JXAvg * FDX1 + JYAvg * FDY1) * R(0.5) + Tau0SpaVar;
  R T2 = (2 * ESN2 + 1 * (ESN1 + ESN3)) * MsFacR -
              c0 * (C00 * (FDX2 * E0XGrad2A + FDY2 * E0YGrad2A)) -
              c1 * (A00pB00 * (FDX2 * E1XGrad2A + FDY2 * E1YGrad2A)) +
              (JXAvg * FDX2 + JYAvg * FDY2) * R(0.5) + Tau0SpaVar;
  R T3 = (2 * ESN3 + 1 * (ESN1 + ESN2)) * MsFacR -
              c0 * (C00 * (FDX3 * E0XGrad2A + FDY3 * E0YGrad2A)) -
              c1 * (A00pB00 * (FDX3 * E1XGrad2A + FDY3 * E1YGrad2A)) +
              (JXAvg * FDX3 + JYAvg * FDY3) * R(0.5) + Tau0SpaVar;
  R nc = (R)NCEle;
  const R o[3] = {T1 * nc, T2 * nc, T3 * nc};
  warp_store_k<3>(reinterpret_cast<R *>(c.ebuf) + 3 * (size_t)e0, o, nvalid, sh[threadIdx.x >> 5]);
}

// GWCE_LV gather (element order) fused with gwce.F:1622-1631.
template <class R>
__global__ void k_rhs_gather(adc_ctx c) {
  griddep_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.np) return;
  const R *eb = reinterpret_cast<const R *>(c.ebuf);
  R v = R(0.0);
  const int q0 = c.n2e_ptr[i], q1 = c.n2e_ptr[i + 1];
  for (int qc = q0; qc < q1; qc += kGatherChunk) {
    int ek[kGatherChunk];
    R x[kGatherChunk];
#pragma unroll
    for (int k = 0; k < kGatherChunk; ++k) if (qc + k < q1) ek[k] = c.n2e[qc + k];
#pragma unroll
    for (int k = 0; k < kGatherChunk; ++k) if (qc + k < q1) x[k] = eb[ek[k]];
#pragma unroll
    for (int k = 0; k < kGatherChunk; ++k) if (qc + k < q1) v = v + x[k];
  }
  c.gwce_lv[i] = (double)v;
  c.eta1[i] = c.eta2[i];
  c.h1[i] = c.h2[i];
  c.eta2[i] = 0.0;
}

// gwce.F:1638-1651 periodic elevation BC and :1846-1850 load-vector rows.
__global__ void k_eta_bc(adc_ctx c, const adc_step_t *steps, const Flags *flags) {
  griddep_wait();
  int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= c.neta) return;
  const adc_step_t st = steps[flags->cursor];
  int b = c.nbd[I];
  double e2 = 0.0;   // ETA2 was zeroed in k_rhs_gather
  for (int J = 0; J < c.nbfr; ++J) {
    int NCYC = 0;
    if (c.per[J] != 0.0) NCYC = (int)(st.timeh / c.per[J]);
    double ARGJ = c.amig[J] * (st.timeh - NCYC * c.per[J]) + c.face[J];
    double RFF = c.ff[J] * st.rampelev;
    double ARG = ARGJ - c.efa[J + (size_t)c.nbfr * I];
    e2 = e2 + c.emo[J + (size_t)c.nbfr * I] * RFF * cos(ARG);
  }
  if (c.eser_on) {   // non-periodic elevations, gwce.F:1668-1673
    const SeriesState &ss = c.sstate[0];
    const size_t r1 = (size_t)ss.k * c.neta, r2 = r1 + c.neta;
    e2 = e2 + st.rampelev * (c.eser[r1 + I] + ss.ratio * (c.eser[r2 + I] - c.eser[r1 + I]));
  }
  c.eta2[b] = e2;
  double es = e2 - c.eta1[b];
  c.etas[b] = es;
  c.gwce_lv[b] = es * c.nodecode[b] * flags->ep;
}

// gwce.F:1851-1854 column correction, per affected neighbour in (I, J) order.
__global__ void k_obc_rhs(adc_ctx c) {
  griddep_wait();
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= c.n_obc_rhs_nodes) return;
  int nb = c.obc_rhs_node[r];
  double v = c.gwce_lv[nb];
  for (int q = c.obc_rhs_ptr[r]; q < c.obc_rhs_ptr[r + 1]; ++q)
    v = v - c.etas[c.obc_rhs_b[q]] * c.obccoef[c.obc_rhs_ent[q]];
  c.gwce_lv[nb] = v;
}

template __global__ void k_lhs_elem<double>(adc_ctx, const int *);
template __global__ void k_lhs_elem<float>(adc_ctx, const int *);
template __global__ void k_lhs_gather<double>(adc_ctx, const int *);
template __global__ void k_lhs_gather<float>(adc_ctx, const int *);
template __global__ void k_rhs_elem<double>(adc_ctx);
template __global__ void k_rhs_elem<float>(adc_ctx);
template __global__ void k_rhs_gather<double>(adc_ctx);
template __global__ void k_rhs_gather<float>(adc_ctx);

}  // namespace adc
