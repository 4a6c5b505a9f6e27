// momentum.cu -- Mom_Eqs_New_NC (momentum.F:166-1208): lumped explicit
// non-conservative 2DDI momentum with IBPV lateral stress and corrected
// area integration, land boundary codes 0-19 and the zero normal velocity
// gradient of code 40, Cartesian coordinates.
//
// Two kernels: an element kernel forms the six load-vector contributions
// (momentum.F:298-699); a node kernel gathers them in element order, forms
// the nodal load and the 2x2 LHS (:713-803), applies the velocity boundary
// condition of the node if it has one (:810-862), solves (:1128-1138) and
// writes the fluxes (:1179-1182).  Boundary nodes in ME2GW are distinct,
// so the boundary step is a per-node operation.
#include "adc_internal.cuh"

#include <cfloat>

namespace adc {

// Four 256-thread blocks per SM (64 registers): measured 0.057 ms per
// launch on the surge mesh against 0.062 ms at the compiler's choice (68).
template <class R>
__global__ void __launch_bounds__(256, 4) k_mom_elem(adc_ctx c) {
  griddep_wait();
  __shared__ R sh[kThreads / 32][32 * 6];
  const int e0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31);
  if (e0 >= c.ne) return;
  const int nvalid = min(32, c.ne - e0);
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= c.ne) e = c.ne - 1;   // idle lanes recompute the last element; not stored
  const adc_params_t &p = c.p;
  const R DT = R(p.dt);
  const R THIRD = R(R(1.0)) / R(R(3.0)), GO2 = R(p.g) / R(R(2.0));
  const bool met = p.nws != 0;
  int n1 = c.nm[3 * e], n2 = c.nm[3 * e + 1], n3 = c.nm[3 * e + 2];
  int NCEle = c.nodecode[n1] * c.nodecode[n2] * c.nodecode[n3] * c.noff[e];
  R U1N1 = c.uu1[n1], U1N2 = c.uu1[n2], U1N3 = c.uu1[n3];
  R V1N1 = c.vv1[n1], V1N2 = c.vv1[n2], V1N3 = c.vv1[n3];
  R H1N1 = c.h1[n1], H1N2 = c.h1[n2], H1N3 = c.h1[n3];
  R AreaIE2 = c.areas[e];
  R AreaIE = R(0.5) * AreaIE2;
  R FDX1 = c.fdx[3 * e], FDX2 = c.fdx[3 * e + 1], FDX3 = c.fdx[3 * e + 2];
  R FDY1 = c.fdy[3 * e], FDY2 = c.fdy[3 * e + 1], FDY3 = c.fdy[3 * e + 2];
  R U1Avg = THIRD * (U1N1 + U1N2 + U1N3);
  R V1Avg = THIRD * (V1N1 + V1N2 + V1N3);
  R DU1DXA = (U1N1 * FDX1 + U1N2 * FDX2 + U1N3 * FDX3) * R(0.5);
  R DU1DYA = (U1N1 * FDY1 + U1N2 * FDY2 + U1N3 * FDY3) * R(0.5);
  R DV1DXA = (V1N1 * FDX1 + V1N2 * FDX2 + V1N3 * FDX3) * R(0.5);
  R DV1DYA = (V1N1 * FDY1 + V1N2 * FDY2 + V1N3 * FDY3) * R(0.5);
  R EVMEle = THIRD * (c.evm[n1] + c.evm[n2] + c.evm[n3]);
  R al = c.alphal[e];
  R B11 = al * c.eta1[n1], B21 = al * c.eta2[n1];
  R B12 = al * c.eta1[n2], B22 = al * c.eta2[n2];
  R B13 = al * c.eta1[n3], B23 = al * c.eta2[n3];
  if (met) {
    if constexpr (sizeof(R) == 4) {
      // only gradients of B are used: FP32 carries the pressure's deviation
      // from the background, not the ~10 m total
      const double pb = p.prbckgrnd_mh2o;
      B11 = B11 + R(c.pr1[n1] - pb); B21 = B21 + R(c.pr2[n1] - pb);
      B12 = B12 + R(c.pr1[n2] - pb); B22 = B22 + R(c.pr2[n2] - pb);
      B13 = B13 + R(c.pr1[n3] - pb); B23 = B23 + R(c.pr2[n3] - pb);
    } else {
      B11 = B11 + c.pr1[n1]; B21 = B21 + c.pr2[n1];
      B12 = B12 + c.pr1[n2]; B22 = B22 + c.pr2[n2];
      B13 = B13 + c.pr1[n3]; B23 = B23 + c.pr2[n3];
    }
  }
  R DBTPDX1A, DBTPDX2A, DBTPDY1A, DBTPDY2A;
  if constexpr (sizeof(R) == 4) {
    // barotropic-pressure gradients cancel metre-sized nodal values: FP64,
    // then narrowed
    const double *fx = c.fdx + 3 * e, *fy = c.fdy + 3 * e;
    const double ald = c.alphal[e];
    double b11 = ald * c.eta1[n1], b21 = ald * c.eta2[n1];
    double b12 = ald * c.eta1[n2], b22 = ald * c.eta2[n2];
    double b13 = ald * c.eta1[n3], b23 = ald * c.eta2[n3];
    if (met) {
      b11 += c.pr1[n1]; b21 += c.pr2[n1];
      b12 += c.pr1[n2]; b22 += c.pr2[n2];
      b13 += c.pr1[n3]; b23 += c.pr2[n3];
    }
    DBTPDX1A = R(b11 * fx[0] + b12 * fx[1] + b13 * fx[2]);
    DBTPDX2A = R(b21 * fx[0] + b22 * fx[1] + b23 * fx[2]);
    DBTPDY1A = R(b11 * fy[0] + b12 * fy[1] + b13 * fy[2]);
    DBTPDY2A = R(b21 * fy[0] + b22 * fy[1] + b23 * fy[2]);
  } else {
    DBTPDX1A = B11 * FDX1 + B12 * FDX2 + B13 * FDX3;
    DBTPDX2A = B21 * FDX1 + B22 * FDX2 + B23 * FDX3;
    DBTPDY1A = B11 * FDY1 + B12 * FDY2 + B13 * FDY3;
    DBTPDY2A = B21 * FDY1 + B22 * FDY2 + B23 * FDY3;
  }
  R DBTPDXA = R(0.5) * (DBTPDX1A + DBTPDX2A);   // Cfac1 = Cfac2 = 1
  R DBTPDYA = R(0.5) * (DBTPDY1A + DBTPDY2A);
  R ADVX = U1Avg * DU1DXA + V1Avg * DU1DYA;
  R ADVY = U1Avg * DV1DXA + V1Avg * DV1DYA;
  R DU1DX = DU1DXA / AreaIE, DU1DY = DU1DYA / AreaIE;
  R DV1DX = DV1DXA / AreaIE, DV1DY = DV1DYA / AreaIE;
  R EH1 = EVMEle * H1N1, EH2 = EVMEle * H1N2, EH3 = EVMEle * H1N3;
  R nc = (R)NCEle;
  R fct = nc * DT;
  R ax = -p.ifnlct * ADVX - GO2 * DBTPDXA - R(0.0);
  R ay = -p.ifnlct * ADVY - GO2 * DBTPDYA - R(0.0);
  R o[6];
  o[0] = fct * (ax - (R(1.5) * ((EH1 * DU1DX) * FDX1 + (EH1 * DU1DY) * FDY1)) / H1N1);
  o[1] = fct * (ax - (R(1.5) * ((EH2 * DU1DX) * FDX2 + (EH2 * DU1DY) * FDY2)) / H1N2);
  o[2] = fct * (ax - (R(1.5) * ((EH3 * DU1DX) * FDX3 + (EH3 * DU1DY) * FDY3)) / H1N3);
  o[3] = fct * (ay - (R(1.5) * ((EH1 * DV1DX) * FDX1 + (EH1 * DV1DY) * FDY1)) / H1N1);
  o[4] = fct * (ay - (R(1.5) * ((EH2 * DV1DX) * FDX2 + (EH2 * DV1DY) * FDY2)) / H1N2);
  o[5] = fct * (ay - (R(1.5) * ((EH3 * DV1DX) * FDX3 + (EH3 * DV1DY) * FDY3)) / H1N3);
  warp_store_k<6>(reinterpret_cast<R *>(c.ebuf) + 6 * (size_t)e0, o, nvalid, sh[threadIdx.x >> 5]);
}

// gfortran's inline NORM2 for TKM(:,i) (scaled sum of squares starting
// from scale = 1), used by adcirc_norm2 (global.F:1502-1515).
__device__ double norm2_3(const double *x) {
  double scale = 1.0, result = 0.0;
  for (int i = 0; i < 3; ++i) {
    if (x[i] != 0.0) {
      double absx = fabs(x[i]);
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
  return scale * sqrt(result);
}

template <class R>
__global__ void k_mom_node(adc_ctx c) {
  griddep_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.np) return;
  const adc_params_t &p = c.p;
  const double DTO2 = p.dt / 2.0;
  const R *eb = reinterpret_cast<const R *>(c.ebuf);
  R mxr = R(0.0), myr = R(0.0);
  const int q0 = c.n2e_ptr[i], q1 = c.n2e_ptr[i + 1];
  for (int qc = q0; qc < q1; qc += kGatherChunk) {
    int ek[kGatherChunk];
    R xa[kGatherChunk], xb[kGatherChunk];
#pragma unroll
    for (int k = 0; k < kGatherChunk; ++k) if (qc + k < q1) ek[k] = c.n2e[qc + k];
#pragma unroll
    for (int k = 0; k < kGatherChunk; ++k)
      if (qc + k < q1) {
        int e = ek[k] / 3, kk = ek[k] - 3 * e;
        xa[k] = eb[6 * (size_t)e + kk];
        xb[k] = eb[6 * (size_t)e + 3 + kk];
      }
#pragma unroll
    for (int k = 0; k < kGatherChunk; ++k)
      if (qc + k < q1) {
        mxr = mxr + xa[k];
        myr = myr + xb[k];
      }
  }
  double mx = (double)mxr, my = (double)myr;
  int NCI = c.nodecode[i];
  double ta = c.totalarea[i];
  if (ta != 0.0) {
    mx = mx / ta;
    my = my / ta;
  }
  double uu1 = c.uu1[i], vv1 = c.vv1[i];
  double WSX = 0.0, WSY = 0.0;
  if (p.nws != 0) {
    WSX = DTO2 * p.ifwind * (c.wsx1[i] / c.h1[i] + c.wsx2[i] / c.h2[i]);
    WSY = DTO2 * p.ifwind * (c.wsy1[i] / c.h1[i] + c.wsy2[i] / c.h2[i]);
  }
  const double *tkm = c.tkm + 3 * i;
  double VXX = DTO2 * (tkm[0] + 0.0);
  double VYY = DTO2 * (tkm[1] + 0.0);
  double CorifA = c.corif[i];
  double VXY = DTO2 * (tkm[2] - CorifA);
  double VYX = DTO2 * (tkm[2] + CorifA);
  mx = NCI * (mx + WSX + (1.0 - VXX) * uu1 - VXY * vv1);
  my = NCI * (my + WSY + (1.0 - VYY) * vv1 - VYX * uu1);
  double a1 = 1.0 + VXX * NCI, a2 = 1.0 + VYY * NCI, a3 = VXY * NCI, a4 = VYX * NCI;
  int me = c.me_of_node[i];
  if (me >= 0) {
    int lb = c.me_lbc[me];
    double csi = c.me_csi[me], sii = c.me_sii[me];
    const double qn2 = c.qn[2 * c.nvel + c.me_i[me]];   // zero on land boundaries
    if (lb >= 0 && lb <= 9) {
      double VelNorm = -qn2 / c.h2[i];
      if (fabs(norm2_3(tkm) - sqrt(2.0) * c.tk[i]) < DBL_EPSILON) {
        mx = (sii * mx - csi * my - VelNorm * a3) * NCI;
        my = VelNorm * a1 * NCI;
        a3 = -csi * a1;
        a4 = -a3;
        a1 = sii * a1;
        a2 = a1;
      } else {
        mx = (sii * mx - csi * my) * NCI;
        my = VelNorm * NCI;
        double n1 = a1 * sii - a4 * csi;
        double n3 = a3 * sii - a2 * csi;
        a1 = n1;
        a3 = n3;
        a4 = csi;
        a2 = sii;
      }
    }
    if (lb >= 10 && lb <= 19) {
      double VelNorm = -qn2 / c.h2[i];
      mx = 0.0 * NCI;
      my = VelNorm * NCI;
      a1 = sii;
      a3 = -csi;
      a4 = csi;
      a2 = sii;
    }
    if (lb == 41) {
      // zero normal velocity gradient by a Galerkin normal derivative over
      // the ring's elements (momentum.F:864-933), from the old velocities
      double r1 = 0.0, r2 = 0.0, lhs = 0.0;
      for (int q = c.me41_ptr[me]; q < c.me41_ptr[me + 1]; ++q) {
        const int nm2 = c.me41_tri[3 * q], nm3 = c.me41_tri[3 * q + 1], e = c.me41_tri[3 * q + 2];
        if (e < 0) continue;
        const int NCEle = NCI * c.nodecode[nm2] * c.nodecode[nm3] * c.noff[e];
        if (NCEle == 0) continue;
        const double FDX1 = c.fdx[3 * e] * 1.0, FDX2 = c.fdx[3 * e + 1] * 1.0, FDX3 = c.fdx[3 * e + 2] * 1.0;
        const double FDY1 = c.fdy[3 * e] * 1.0, FDY2 = c.fdy[3 * e + 1] * 1.0, FDY3 = c.fdy[3 * e + 2] * 1.0;
        r1 = r1 - (csi * FDX2 + sii * FDY2) * c.uu1[nm2] - (csi * FDX3 + sii * FDY3) * c.uu1[nm3];
        r2 = r2 - (csi * FDX2 + sii * FDY2) * c.vv1[nm2] - (csi * FDX3 + sii * FDY3) * c.vv1[nm3];
        lhs = lhs + csi * FDX1 + sii * FDY1;
      }
      if (NCI == 0) {
        mx = 0.0;
        my = 0.0;
      } else {
        mx = r1 / lhs;
        my = r2 / lhs;
      }
      a1 = 1.0;
      a2 = 1.0;
      a3 = 0.0;
      a4 = 0.0;
    }
  }
  c.mom_x[i] = mx;
  c.mom_y[i] = my;
  double DDU = a1 * a2 - a3 * a4;
  double u2 = (mx * a2 - my * a3) / DDU;
  double v2 = (my * a1 - mx * a4) / DDU;
  c.uu2[i] = u2;
  c.vv2[i] = v2;
  double h2 = c.h2[i];
  c.qx2[i] = u2 * h2;
  c.qy2[i] = v2 * h2;
}

// Zero normal velocity gradient (IBTYPE 40), momentum.F:1157-1174: after
// the nodal solve each such boundary node takes the velocity interpolated
// at its fictitious interior node, then its fluxes (:1179-1182).  The
// entries go in ME2GW order on one thread, since an entry's element may
// hold a node an earlier entry has just set.
__global__ void k_mom_zng(adc_ctx c) {
  griddep_wait();
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int k = 0; k < c.n_zng; ++k) {
    const int n = c.zng_node[k], e = c.zng_ele[k];
    const int NM1 = c.nm[3 * e], NM2 = c.nm[3 * e + 1], NM3 = c.nm[3 * e + 2];
    const int NCEle = c.nodecode[NM1] * c.nodecode[NM2] * c.nodecode[NM3] * c.noff[e];
    const double f1 = c.zng_f[3 * k], f2 = c.zng_f[3 * k + 1], f3 = c.zng_f[3 * k + 2];
    const double u = NCEle * (c.uu2[NM1] * f1 + c.uu2[NM2] * f2 + c.uu2[NM3] * f3);
    const double v = NCEle * (c.vv2[NM1] * f1 + c.vv2[NM2] * f2 + c.vv2[NM3] * f3);
    c.uu2[n] = u;
    c.vv2[n] = v;
    c.qx2[n] = u * c.h2[n];
    c.qy2[n] = v * c.h2[n];
  }
}

int launch_momentum(adc_ctx *c) {
  kmark(c, KS_MOM_ELEM, 0);
  if (f32_momentum(c)) {   // FP32 element terms and their gather
    launch_k(k_mom_elem<float>, nblk(c->ne), kThreads, c->stream, *c);
    kmark(c, KS_MOM_ELEM, 1);
    kmark(c, KS_MOM_NODE, 0);
    launch_k(k_mom_node<float>, nblk(c->np), kThreads, c->stream, *c);
  } else {
    launch_k(k_mom_elem<double>, nblk(c->ne), kThreads, c->stream, *c);
    kmark(c, KS_MOM_ELEM, 1);
    kmark(c, KS_MOM_NODE, 0);
    launch_k(k_mom_node<double>, nblk(c->np), kThreads, c->stream, *c);
  }
  if (c->n_zng > 0) {
    launch_k(k_mom_zng, 1, 32, c->stream, *c);
    c->launches++;
  }
  kmark(c, KS_MOM_NODE, 1);
  c->launches += 2;
  return ADC_OK;
}

template __global__ void k_mom_elem<double>(adc_ctx);
template __global__ void k_mom_elem<float>(adc_ctx);
template __global__ void k_mom_node<double>(adc_ctx);
template __global__ void k_mom_node<float>(adc_ctx);

}  // namespace adc
