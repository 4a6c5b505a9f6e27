/*
 * mesh_prep.cpp -- one-time host-side mesh and boundary tables.
 *
 * In the reference these tables are built by the Fortran host during
 * ADCIRC_Init and live in module MESH / BOUNDARIES; the hot path only reads
 * them.  A Fortran host binds its own arrays through adc_gpu_bind(); a host
 * without the reference's initialisation (the Python harness of this
 * package) builds the same tables here.  Cartesian coordinates (ICS = 1).
 *
 *   adc_mesh_geometry      mesh.F:1558-1664   FDXE, FDYE, AREAS, CCW order
 *   adc_mesh_mnei          mesh.F:1712-1726   MNEI = max element count + 2
 *   adc_mesh_neighb        mesh.F:3089-3318   NeiTab sorted by angle, NNeigh
 *   adc_mesh_csr_positions mesh.F:5261-5282   CSR_POSITION(NE,3,2)
 *   adc_boundary_setup     mesh.F:2100-2800   NBV, LBCODEI, CSII, SIII, ME2GW, BNDLEN2O3
 *   adc_zng_setup          mesh.F:2434-2512   NEleZNG, ZNGIF1-3 (IBTYPE 40)
 *   adc_mesh_neitabele     mesh.F:3110-3131, 3248-3283   NeiTabEle
 *
 * All arrays use the reference layout: column-major, 1-based node numbers.
 */
#include "../../include/adcgpu.h"

#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>

namespace {
constexpr double kPi = 3.141592653589793;
constexpr double kRad2Deg = 180.0 / kPi;
}

extern "C" {

int adc_mesh_geometry(int np, int ne, const double *x, const double *y, int *nm,
                      double *fdxe, double *fdye, double *areas) {
  if (np <= 0 || ne <= 0) return ADC_ERR_ARG;
  for (int i = 0; i < ne; ++i) {
    int *n1 = &nm[i], *n2 = &nm[i + (size_t)ne], *n3 = &nm[i + 2 * (size_t)ne];
    for (int pass = 0; pass < 2; ++pass) {
      if (*n1 < 1 || *n1 > np || *n2 < 1 || *n2 > np || *n3 < 1 || *n3 > np) return ADC_ERR_ARG;
      double X1 = x[*n1 - 1], X2 = x[*n2 - 1], X3 = x[*n3 - 1];
      double Y1 = y[*n1 - 1], Y2 = y[*n2 - 1], Y3 = y[*n3 - 1];
      double X2mX1 = X2 - X1, X3mX2 = X3 - X2, X1mX3 = X1 - X3;
      double Y2mY1 = Y2 - Y1, Y3mY2 = Y3 - Y2, Y1mY3 = Y1 - Y3;
      fdxe[3 * (size_t)i + 0] = -Y3mY2;
      fdxe[3 * (size_t)i + 1] = -Y1mY3;
      fdxe[3 * (size_t)i + 2] = -Y2mY1;
      fdye[3 * (size_t)i + 0] = X3mX2;
      fdye[3 * (size_t)i + 1] = X1mX3;
      fdye[3 * (size_t)i + 2] = X2mX1;
      areas[i] = (X1mX3) * (-Y3mY2) + (X3mX2) * (Y1mY3);
      if (areas[i] < 0.0 && pass == 0) {
        std::swap(*n2, *n3); /* reorder and start again, mesh.F:1649-1652 */
      } else {
        break;
      }
    }
    if (areas[i] <= 0.0) return ADC_ERR_MESH;
  }
  return ADC_OK;
}

int adc_mesh_mnei(int np, int ne, const int *nm) {
  std::vector<int> cnt(np, 0);
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < ne; ++i) {
      int n = nm[i + (size_t)ne * k];
      if (n < 1 || n > np) return -1;
      cnt[n - 1]++;
    }
  int mx = 0;
  for (int c : cnt) mx = std::max(mx, c);
  return mx + 2;
}

int adc_mesh_neighb(int np, int ne, int mnei, const double *x, const double *y,
                    const int *nm, int *nneigh, int *neitab, int *neimax_out) {
  std::vector<int> etmp((size_t)np * mnei, 0);
  std::fill(nneigh, nneigh + np, 0);
  std::fill(neitab, neitab + (size_t)np * mnei, 0);
  auto NT = [&](int node, int j) -> int & { return neitab[(node - 1) + (size_t)np * (j - 1)]; };
  auto ET = [&](int node, int j) -> int & { return etmp[(node - 1) + (size_t)np * (j - 1)]; };
  auto add_pair = [&](int a, int b, int elem) -> bool {
    bool found = false;
    for (int j = 1; j <= nneigh[a - 1]; ++j)
      if (b == NT(a, j)) { found = true; break; }
    if (!found) {
      nneigh[a - 1]++;
      nneigh[b - 1]++;
      if (nneigh[a - 1] > mnei - 1 || nneigh[b - 1] > mnei - 1) return false;
      NT(a, nneigh[a - 1]) = b;
      NT(b, nneigh[b - 1]) = a;
      ET(a, nneigh[a - 1]) = elem;
      ET(b, nneigh[b - 1]) = elem;
    }
    return true;
  };
  for (int n = 1; n <= ne; ++n) {
    int nn1 = nm[(n - 1)], nn2 = nm[(n - 1) + (size_t)ne], nn3 = nm[(n - 1) + 2 * (size_t)ne];
    if (!add_pair(nn1, nn2, n) || !add_pair(nn1, nn3, n) || !add_pair(nn2, nn3, n))
      return ADC_ERR_MESH;
  }
  std::vector<double> angle(mnei);
  std::vector<int> neitem(mnei);
  for (int i = 1; i <= np; ++i) {
    int nn = nneigh[i - 1];
    for (int j = 1; j <= nn; ++j) {
      neitem[j - 1] = NT(i, j);
      int ej = ET(i, j);
      /* element-local vertex coordinates (EXV/EYV); Cartesian: X/Y */
      double delx = x[neitem[j - 1] - 1] - x[i - 1];
      double dely = y[neitem[j - 1] - 1] - y[i - 1];
      (void)ej;
      double dist = std::sqrt(delx * delx + dely * dely);
      if (dist == 0.0) return ADC_ERR_MESH;
      if (dely != 0.0) {
        angle[j - 1] = kRad2Deg * std::acos(delx / dist);
        if (dely > 0.0) angle[j - 1] = 360.0 - angle[j - 1];
      }
      if (dely == 0.0) {
        if (delx > 0.0) angle[j - 1] = 0.0;
        if (delx < 0.0) angle[j - 1] = 180.0;
      }
    }
    double anglemore = -1.0;
    int jlow = 1;
    for (int jj = 1; jj <= nn; ++jj) {
      double anglelow = 400.0;
      for (int j = 1; j <= nn; ++j) {
        if (angle[j - 1] < anglelow && angle[j - 1] > anglemore) {
          anglelow = angle[j - 1];
          jlow = j;
        }
      }
      NT(i, jj + 1) = neitem[jlow - 1];
      anglemore = anglelow;
    }
    NT(i, 1) = i;
    nneigh[i - 1] = nn + 1;
  }
  int neimax = 0;
  for (int n = 0; n < np; ++n) neimax = std::max(neimax, nneigh[n]);
  if (neimax_out) *neimax_out = neimax;
  return ADC_OK;
}

int adc_mesh_csr_positions(int np, int ne, int mnei, const int *nm, const int *neitab,
                           int neimax, int *csr_position) {
  auto NT = [&](int node, int j) { return neitab[(node - 1) + (size_t)np * (j - 1)]; };
  auto CP = [&](int i, int k, int l) -> int & {
    return csr_position[(i - 1) + (size_t)ne * ((k - 1) + 3 * (l - 1))];
  };
  if (neimax > mnei) return ADC_ERR_ARG;
  for (int i = 1; i <= ne; ++i) {
    int nn1 = nm[i - 1], nn2 = nm[(i - 1) + (size_t)ne], nn3 = nm[(i - 1) + 2 * (size_t)ne];
    for (int k = 1; k <= 3; ++k) for (int l = 1; l <= 2; ++l) CP(i, k, l) = 0;
    for (int jn = 2; jn <= neimax; ++jn) {
      if (NT(nn1, jn) == nn2) CP(i, 1, 1) = jn;
      if (NT(nn1, jn) == nn3) CP(i, 1, 2) = jn;
      if (NT(nn2, jn) == nn1) CP(i, 2, 1) = jn;
      if (NT(nn2, jn) == nn3) CP(i, 2, 2) = jn;
      if (NT(nn3, jn) == nn1) CP(i, 3, 1) = jn;
      if (NT(nn3, jn) == nn2) CP(i, 3, 2) = jn;
    }
    for (int k = 1; k <= 3; ++k) for (int l = 1; l <= 2; ++l) if (CP(i, k, l) == 0) return ADC_ERR_MESH;
  }
  return ADC_OK;
}

/*
 * Flow-boundary arrays for external land segments (IBTYPE 0, 10, 20),
 * islands (IBTYPE 1, 11, 21), specified-flow (2, 12, 22), radiation (30),
 * coupled flux/radiation (32), zero-normal-gradient (40, 41),
 * river-radiation (52) and external barrier (3, 13, 23) segments, and the
 * faces of internal barriers (4, 24; 5, 25 with pipes): mesh.F processes a barrier segment as
 * its front face and then its back face, each an unclosed segment
 * (mesh.F:2158-2192), so the caller lists the two faces as two segments of
 * the barrier's type, the back face in the reversed order mesh.F gives it,
 * mesh.F:2180-2800.  seg_ptr[k]..seg_ptr[k+1]-1
 * index seg_nodes (1-based node numbers, as listed in fort.14).  Outputs are
 * sized by the caller for nvel_max entries (sum of segment lengths plus one
 * per island for closing).  cos_inner = COS(ANGINN*DEG2RAD).
 */
int adc_boundary_setup(int np, const double *x, const double *y, int nbou,
                       const int *ibtype, const int *seg_ptr, const int *seg_nodes,
                       double cos_inner, int nvel_max, int *nvel_out, int *nbv,
                       int *lbcodei, double *csii, double *siii, int *nvelme_out,
                       int *me2gw, double *bndlen2o3) {
  int jgw = 0, jme = 0;
  /* flow types (specified flow, radiation) take the momentum equation
     where segments overlap (mesh.F:2529-2541, 2555-2566) */
  auto specified_flow = [](int code) {
    return code == 2 || code == 12 || code == 22 || code == 3 || code == 13 || code == 23 ||
           code == 30 || code == 32 || code == 40 || code == 41 || code == 52;
  };
  for (int k = 0; k < nbou; ++k) {
    int t = ibtype[k];
    bool island = (t == 1 || t == 11 || t == 21);
    bool mainland = (t == 0 || t == 10 || t == 20);
    bool flux = specified_flow(t);   /* external boundaries with normal flow or radiation */
    bool barrier_face = (t == 4 || t == 24 || t == 5 || t == 25);
    if (!island && !mainland && !flux && !barrier_face) return ADC_ERR_ARG;
    std::vector<int> nbvv;
    int nvell = seg_ptr[k + 1] - seg_ptr[k];
    if (nvell < 2) return ADC_ERR_ARG;
    nbvv.resize(nvell + 3);
    for (int i = 1; i <= nvell; ++i) nbvv[i] = seg_nodes[seg_ptr[k] + i - 1];
    nbvv[0] = nbvv[1]; /* unclosed external */
    /* a two-node island closed here gets its normal from the node pair
       itself (FLG_IBLEN2, mesh.F:2231, 2421-2424) */
    bool iblen2 = false;
    if (island && nbvv[nvell] != nbvv[1]) {
      iblen2 = (nvell == 2);
      nvell = nvell + 1;
      nbvv.resize(nvell + 3);
      nbvv[nvell] = nbvv[1];
    }
    if (nbvv[nvell] == nbvv[1]) nbvv[0] = nbvv[nvell - 1]; /* closed */
    nbvv[nvell + 1] = nbvv[nvell];
    double theta1 = 0, cross1 = 0, costheta1 = 0;
    for (int i = 1; i <= nvell; ++i) {
      if (jgw >= nvel_max) return ADC_ERR_ARG;
      jgw = jgw + 1;
      int nbvi = nbvv[i], nbvj = nbvv[i + 1], nbvk = nbvv[i - 1];
      if (nbvi < 1 || nbvi > np || nbvj < 1 || nbvj > np || nbvk < 1 || nbvk > np) return ADC_ERR_ARG;
      nbv[jgw - 1] = nbvi;
      double xgj = x[nbvj - 1], xgi = x[nbvi - 1], xgk = x[nbvk - 1];
      double ygj = y[nbvj - 1], ygi = y[nbvi - 1], ygk = y[nbvk - 1];
      double theta = 0, cross = 0, costheta = 0;
      bool calc = true;
      if (i == 1 && nbvv[1] == nbvv[0]) {
        theta = -9999999.0;
        cross = 0.0;
        costheta = cos_inner;
        calc = false;
      }
      if (i == nvell) {
        theta = theta1;
        cross = cross1;
        costheta = costheta1;
        calc = false;
      }
      if (calc) {
        double vl1x = xgk - xgi, vl1y = ygk - ygi, vl2x = xgj - xgi, vl2y = ygj - ygi;
        double dotvec = vl1x * vl2x + vl1y * vl2y;
        double vecnorm = (std::sqrt(vl1x * vl1x + vl1y * vl1y)) * (std::sqrt(vl2x * vl2x + vl2y * vl2y));
        costheta = dotvec / vecnorm;
        if (costheta > 1.0) costheta = 1.0;
        if (costheta < -1.0) costheta = -1.0;
        theta = kRad2Deg * std::acos(costheta);
        cross = -vl1x * vl2y + vl2x * vl1y;
        if (cross < 0) theta = 360.0 - theta;
      }
      if (i == 1) { theta1 = theta; cross1 = cross; costheta1 = costheta; }
      lbcodei[jgw - 1] = t;
      if (costheta > cos_inner && cross > 0.0) {
        if (t == 0) lbcodei[jgw - 1] = 10;
        if (t == 1) lbcodei[jgw - 1] = 11;
        if (t == 2) lbcodei[jgw - 1] = 12;
        if (t == 3) lbcodei[jgw - 1] = 13;
      }
      /* 2/3 of the segment to the next node, mesh.F:2301-2303 (zero after
         the last node of an unclosed segment) */
      if (bndlen2o3) {
        const double delx = xgj - xgi, dely = ygj - ygi;
        bndlen2o3[jgw - 1] = 2.0 * (std::sqrt(delx * delx + dely * dely)) / 3.0;
      }
      if (iblen2) { xgj = xgi; ygj = ygi; }
      double xl = std::sqrt((xgk - xgj) * (xgk - xgj) + (ygk - ygj) * (ygk - ygj));
      csii[jgw - 1] = 1.0 * (ygj - ygk) / xl;
      siii[jgw - 1] = (xgk - xgj) / xl;
      /* momentum-equation key, mesh.F:2516-2568: a node shared by two
         segments keeps one entry, the specified-flow one if there is one */
      if (i == 1) {
        if (jgw == 1) { jme++; me2gw[jme - 1] = jgw; }
        if (jgw != 1 && nbv[jgw - 1] != nbv[jgw - 2]) { jme++; me2gw[jme - 1] = jgw; }
        if (jgw != 1 && nbv[jgw - 1] == nbv[jgw - 2] && specified_flow(lbcodei[jgw - 1]) && jme > 0)
          me2gw[jme - 1] = jgw;
      }
      if (i > 1 && i < nvell) { jme++; me2gw[jme - 1] = jgw; }
      if (i == nvell) {
        if (nbv[jgw - 1] != nbvv[1] && nbv[jgw - 1] != nbv[0]) { jme++; me2gw[jme - 1] = jgw; }
        if (nbvv[i] == nbv[0] && specified_flow(lbcodei[jgw - 1])) me2gw[0] = jgw;
      }
    }
  }
  *nvel_out = jgw;
  *nvelme_out = jme;
  return ADC_OK;
}


/*
 * NeiTabEle (NEIGHB, mesh.F:3110-3131, 3248-3283): for each node, its
 * elements in the order of its NeiTab ring: going round the ring, the
 * element with vertices (node, next neighbour, this neighbour) in
 * counter-clockwise order, first match in element-number order; entries
 * without such an element are skipped, so the list is packed from the
 * front (zeros after it).  neitabele is NeiTabEle(NP,MNEI), 1-based.
 */
int adc_mesh_neitabele(int np, int ne, int mnei, const int *nm, const int *nneigh,
                       const int *neitab, int *neitabele) {
  if (np <= 0 || ne <= 0 || mnei < 3) return ADC_ERR_ARG;
  std::vector<std::vector<int>> around(np);
  for (int e = 0; e < ne; ++e)
    for (int k = 0; k < 3; ++k) {
      const int v = nm[e + (size_t)ne * k] - 1;
      if (v < 0 || v >= np) return ADC_ERR_ARG;
      around[v].push_back(e + 1);
    }
  std::memset(neitabele, 0, sizeof(int) * (size_t)np * mnei);
  for (int i = 0; i < np; ++i) {
    std::vector<int> cand = around[i];
    const int nn = nneigh[i];
    if (nn > mnei) return ADC_ERR_ARG;
    int found = 0;
    for (int j = 2; j <= nn; ++j) {
      const int nn1 = i + 1;
      const int nn3 = neitab[i + (size_t)np * (j - 1)];
      const int nn2 = j != nn ? neitab[i + (size_t)np * j] : neitab[i + (size_t)np * 1];
      for (int &e : cand) {
        if (e == 0) continue;
        const int a = nm[e - 1], b = nm[e - 1 + (size_t)ne], c = nm[e - 1 + 2 * (size_t)ne];
        // the element's vertices rotated to start at the node
        const int r2 = a == nn1 ? b : (b == nn1 ? c : a);
        const int r3 = a == nn1 ? c : (b == nn1 ? a : b);
        if (r2 == nn2 && r3 == nn3) {
          if (found >= mnei) return ADC_ERR_MESH;
          neitabele[i + (size_t)np * found] = e;
          ++found;
          e = 0;
          break;
        }
      }
    }
  }
  return ADC_OK;
}

/*
 * Fictitious interior nodes of the zero-normal-velocity-gradient entries
 * (IBTYPE 40), mesh.F:2434-2512.  For each such boundary entry: a point
 * inward along the entry's normal (CSII, SIII) at 1.001 times the distance
 * to its farthest NeiTab neighbour; the element holding it, taken as the
 * one whose three sub-triangle areas add up closest to its own area (the
 * first such element in element order); and the point's linear
 * interpolation factors in that element.  Entries of other types get
 * NEleZNG = 0.  All node and element numbers are 1-based.
 */
int adc_zng_setup(int np, int ne, const double *x, const double *y, const int *nm, int mnei,
                  const int *nneigh, const int *neitab, const double *areas, int nvel,
                  const int *nbv, const int *lbcodei, const double *csii, const double *siii,
                  int *nelezng, double *zngif1, double *zngif2, double *zngif3) {
  if (np <= 0 || ne <= 0 || nvel < 0) return ADC_ERR_ARG;
  auto N = [&](int ie, int k) { return nm[ie + (size_t)ne * k] - 1; };
  for (int j = 0; j < nvel; ++j) {
    nelezng[j] = 0;
    zngif1[j] = zngif2[j] = zngif3[j] = 0.0;
    if (lbcodei[j] != 40) continue;
    const int i = nbv[j] - 1;
    if (i < 0 || i >= np) return ADC_ERR_ARG;
    double dist = 0.0;
    for (int q = 2; q <= nneigh[i] && q <= mnei; ++q) {
      const int nb = neitab[i + (size_t)np * (q - 1)] - 1;
      if (nb < 0 || nb >= np) return ADC_ERR_ARG;
      const double dx = x[nb] - x[i], dy = y[nb] - y[i];
      const double d = std::sqrt(dx * dx + dy * dy);
      if (dist < d) dist = d;
    }
    dist = 1.001 * dist;
    const double x4 = x[i] - dist * csii[j], y4 = y[i] - dist * siii[j];
    double best = (double)1.0e25f;   /* AEMIN = 1.0E+25, a default-kind REAL */
    int ele = -1;
    for (int e = 0; e < ne; ++e) {
      const int a = N(e, 0), b = N(e, 1), c = N(e, 2);
      const double x1 = x[a], x2 = x[b], x3 = x[c], y1 = y[a], y2 = y[b], y3 = y[c];
      const double A1 = (x4 - x3) * (y2 - y3) + (x2 - x3) * (y3 - y4);
      const double A2 = (x4 - x1) * (y3 - y1) - (y4 - y1) * (x3 - x1);
      const double A3 = (y4 - y1) * (x2 - x1) - (x4 - x1) * (y2 - y1);
      const double AA = std::fabs(A1) + std::fabs(A2) + std::fabs(A3);
      const double AE = std::fabs(AA - areas[e]) / areas[e];
      if (AE < best) {
        best = AE;
        ele = e;
      }
    }
    if (ele < 0) return ADC_ERR_MESH;
    const int a = N(ele, 0), b = N(ele, 1), c = N(ele, 2);
    const double x1 = x[a], x2 = x[b], x3 = x[c], y1 = y[a], y2 = y[b], y3 = y[c];
    nelezng[j] = ele + 1;
    zngif1[j] = ((x4 - x3) * (y2 - y3) + (x2 - x3) * (y3 - y4)) / areas[ele];
    zngif2[j] = ((x4 - x1) * (y3 - y1) - (y4 - y1) * (x3 - x1)) / areas[ele];
    zngif3[j] = (-(x4 - x1) * (y2 - y1) + (y4 - y1) * (x2 - x1)) / areas[ele];
  }
  return ADC_OK;
}
} /* extern "C" */

extern "C" {
/*
 * Cold-start wet/dry state, cstart.F:1332-1427 (non-subgrid branch), then
 * totalAreaCalc, mesh.F:3360-3400.  ETA2 comes in as the initial
 * elevation; nodes with DP+ETA2 <= H0 and landlocked nodes start dry with
 * ETA2 = H0 - DP; ETA1 = ETA2.
 */
int adc_coldstart(int np, int ne, int nolifa, double h0, const double *dp, const int *nm,
                  const double *areas, double *eta1, double *eta2, int *nnodecode,
                  int *nodecode, int *noff, int *mju, double *totalarea) {
  if (np <= 0 || ne <= 0) return ADC_ERR_ARG;
  auto N = [&](int ie, int k) { return nm[ie + (size_t)ne * k] - 1; };
  for (int i = 0; i < np; ++i) nnodecode[i] = 1;
  for (int i = 0; i < ne; ++i) noff[i] = 1;
  if (nolifa == 2) {
    for (int i = 0; i < np; ++i)
      if (dp[i] + eta2[i] <= h0) nnodecode[i] = 0;
    std::vector<int> m(np, 0);
    for (int ie = 0; ie < ne; ++ie) {
      int a = N(ie, 0), b = N(ie, 1), c = N(ie, 2);
      int nc = nnodecode[a] * nnodecode[b] * nnodecode[c] * noff[ie];
      m[a] += nc; m[b] += nc; m[c] += nc;
    }
    for (int i = 0; i < np; ++i)
      if (nnodecode[i] == 1 && m[i] == 0) nnodecode[i] = 0;
    for (int i = 0; i < np; ++i)
      if (nnodecode[i] == 0) eta2[i] = h0 - dp[i];
  }
  for (int i = 0; i < np; ++i) eta1[i] = eta2[i];
  for (int i = 0; i < np; ++i) { mju[i] = 0; totalarea[i] = 0.0; nodecode[i] = nnodecode[i]; }
  for (int ie = 0; ie < ne; ++ie) {
    int a = N(ie, 0), b = N(ie, 1), c = N(ie, 2);
    int nc = nodecode[a] * nodecode[b] * nodecode[c] * noff[ie];
    mju[a] += nc; mju[b] += nc; mju[c] += nc;
    double ae = nc * areas[ie] / 2.0;
    totalarea[a] = totalarea[a] + ae;
    totalarea[b] = totalarea[b] + ae;
    totalarea[c] = totalarea[c] + ae;
  }
  for (int i = 0; i < np; ++i) if (mju[i] == 0) mju[i] = 1;
  return ADC_OK;
}
} /* extern "C" */
