// momentum.cu -- Mom_Eqs_New_NC (momentum.F:166-1208): lumped explicit
// non-conservative 2DDI momentum with IBPV lateral stress and corrected
// area integration, land boundary codes 0-19, Cartesian coordinates.
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

__global__ void k_mom_elem(adc_ctx c) {
  __shared__ double sh[kThreads / 32][32 * 6];
  const int e0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31);
  if (e0 >= c.ne) return;
  const int nvalid = min(32, c.ne - e0);
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= c.ne) e = c.ne - 1;   // idle lanes recompute the last element; not stored
  const adc_params_t &p = c.p;
  const double DT = p.dt;
  const double THIRD = 1.0 / 3.0, GO2 = p.g / 2.0;
  const bool met = p.nws != 0;
  int n1 = c.nm[3 * e], n2 = c.nm[3 * e + 1], n3 = c.nm[3 * e + 2];
  int NCEle = c.nodecode[n1] * c.nodecode[n2] * c.nodecode[n3] * c.noff[e];
  double U1N1 = c.uu1[n1], U1N2 = c.uu1[n2], U1N3 = c.uu1[n3];
  double V1N1 = c.vv1[n1], V1N2 = c.vv1[n2], V1N3 = c.vv1[n3];
  double H1N1 = c.h1[n1], H1N2 = c.h1[n2], H1N3 = c.h1[n3];
  double AreaIE2 = c.areas[e];
  double AreaIE = 0.5 * AreaIE2;
  double FDX1 = c.fdx[3 * e], FDX2 = c.fdx[3 * e + 1], FDX3 = c.fdx[3 * e + 2];
  double FDY1 = c.fdy[3 * e], FDY2 = c.fdy[3 * e + 1], FDY3 = c.fdy[3 * e + 2];
  double U1Avg = THIRD * (U1N1 + U1N2 + U1N3);
  double V1Avg = THIRD * (V1N1 + V1N2 + V1N3);
  double DU1DXA = (U1N1 * FDX1 + U1N2 * FDX2 + U1N3 * FDX3) * 0.5;
  double DU1DYA = (U1N1 * FDY1 + U1N2 * FDY2 + U1N3 * FDY3) * 0.5;
  double DV1DXA = (V1N1 * FDX1 + V1N2 * FDX2 + V1N3 * FDX3) * 0.5;
  double DV1DYA = (V1N1 * FDY1 + V1N2 * FDY2 + V1N3 * FDY3) * 0.5;
  double EVMEle = THIRD * (c.evm[n1] + c.evm[n2] + c.evm[n3]);
  double al = c.alphal[e];
  double B11 = al * c.eta1[n1], B21 = al * c.eta2[n1];
  double B12 = al * c.eta1[n2], B22 = al * c.eta2[n2];
  double B13 = al * c.eta1[n3], B23 = al * c.eta2[n3];
  if (met) {
    B11 = B11 + c.pr1[n1]; B21 = B21 + c.pr2[n1];
    B12 = B12 + c.pr1[n2]; B22 = B22 + c.pr2[n2];
    B13 = B13 + c.pr1[n3]; B23 = B23 + c.pr2[n3];
  }
  double DBTPDX1A = B11 * FDX1 + B12 * FDX2 + B13 * FDX3;
  double DBTPDX2A = B21 * FDX1 + B22 * FDX2 + B23 * FDX3;
  double DBTPDY1A = B11 * FDY1 + B12 * FDY2 + B13 * FDY3;
  double DBTPDY2A = B21 * FDY1 + B22 * FDY2 + B23 * FDY3;
  double DBTPDXA = 0.5 * (DBTPDX1A + DBTPDX2A);   // Cfac1 = Cfac2 = 1
  double DBTPDYA = 0.5 * (DBTPDY1A + DBTPDY2A);
  double ADVX = U1Avg * DU1DXA + V1Avg * DU1DYA;
  double ADVY = U1Avg * DV1DXA + V1Avg * DV1DYA;
  double DU1DX = DU1DXA / AreaIE, DU1DY = DU1DYA / AreaIE;
  double DV1DX = DV1DXA / AreaIE, DV1DY = DV1DYA / AreaIE;
  double EH1 = EVMEle * H1N1, EH2 = EVMEle * H1N2, EH3 = EVMEle * H1N3;
  double nc = (double)NCEle;
  double fct = nc * DT;
  double ax = -p.ifnlct * ADVX - GO2 * DBTPDXA - 0.0;
  double ay = -p.ifnlct * ADVY - GO2 * DBTPDYA - 0.0;
  double o[6];
  o[0] = fct * (ax - (1.5 * ((EH1 * DU1DX) * FDX1 + (EH1 * DU1DY) * FDY1)) / H1N1);
  o[1] = fct * (ax - (1.5 * ((EH2 * DU1DX) * FDX2 + (EH2 * DU1DY) * FDY2)) / H1N2);
  o[2] = fct * (ax - (1.5 * ((EH3 * DU1DX) * FDX3 + (EH3 * DU1DY) * FDY3)) / H1N3);
  o[3] = fct * (ay - (1.5 * ((EH1 * DV1DX) * FDX1 + (EH1 * DV1DY) * FDY1)) / H1N1);
  o[4] = fct * (ay - (1.5 * ((EH2 * DV1DX) * FDX2 + (EH2 * DV1DY) * FDY2)) / H1N2);
  o[5] = fct * (ay - (1.5 * ((EH3 * DV1DX) * FDX3 + (EH3 * DV1DY) * FDY3)) / H1N3);
  warp_store_k<6>(c.ebuf + 6 * (size_t)e0, o, nvalid, sh[threadIdx.x >> 5]);
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

__global__ void k_mom_node(adc_ctx c) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.np) return;
  const adc_params_t &p = c.p;
  const double DTO2 = p.dt / 2.0;
  double mx = 0.0, my = 0.0;
  const int q0 = c.n2e_ptr[i], q1 = c.n2e_ptr[i + 1];
  for (int qc = q0; qc < q1; qc += kGatherChunk) {
    int ek[kGatherChunk];
    double xa[kGatherChunk], xb[kGatherChunk];
#pragma unroll
    for (int k = 0; k < kGatherChunk; ++k) if (qc + k < q1) ek[k] = c.n2e[qc + k];
#pragma unroll
    for (int k = 0; k < kGatherChunk; ++k)
      if (qc + k < q1) {
        int e = ek[k] / 3, kk = ek[k] - 3 * e;
        xa[k] = c.ebuf[6 * (size_t)e + kk];
        xb[k] = c.ebuf[6 * (size_t)e + 3 + kk];
      }
#pragma unroll
    for (int k = 0; k < kGatherChunk; ++k)
      if (qc + k < q1) {
        mx = mx + xa[k];
        my = my + xb[k];
      }
  }
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
    if (lb >= 0 && lb <= 9) {
      double VelNorm = -0.0 / c.h2[i];   // -QN2/H2 with QN2 = 0 (land)
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
      double VelNorm = -0.0 / c.h2[i];
      mx = 0.0 * NCI;
      my = VelNorm * NCI;
      a1 = sii;
      a3 = -csi;
      a4 = csi;
      a2 = sii;
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

int launch_momentum(adc_ctx *c) {
  k_mom_elem<<<nblk(c->ne), kThreads, 0, c->stream>>>(*c);
  k_mom_node<<<nblk(c->np), kThreads, 0, c->stream>>>(*c);
  c->launches += 2;
  return ADC_OK;
}

}  // namespace adc
