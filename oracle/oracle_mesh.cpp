/*
 * oracle_mesh.cpp -- serial restatement of the reference's one-time mesh
 * and boundary tables (mesh.F), for the oracle.
 *
 * TEST INFRASTRUCTURE: the checker's own copy of the static tables, so the
 * oracle never consumes tables built by the library it checks.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU legs load it.
 *
 * Each routine follows the cited reference routine statement by statement
 * (adcirc v56.2.1, src/mesh.F), in Cartesian coordinates (ICS = 1), where
 * the element-local vertex coordinates EXV/EYV are X/Y of the element's
 * nodes (mesh.F:1565-1570) and every spherical factor (SFMX, ...) is 1.
 * The argument lists equal the library's adc_mesh_* / adc_boundary_setup /
 * adc_coldstart so a harness can build a case with either set.
 *
 *   orc_mesh_geometry        mesh.F:1614-1664  FDXE, FDYE, AREAS, NM reorder
 *   orc_mesh_mnei            mesh.F:1716-1731  MNEI = max incident elements + 2
 *   orc_mesh_neighb          mesh.F:3089-3318  NEIGHB: NeiTab by clockwise angle
 *   orc_mesh_csr_positions   mesh.F:5261-5282  compute_csr_positions
 *   orc_boundary_setup       mesh.F:2226-2568  NBV, LBCODEI, CSII, SIII, ME2GW, BNDLEN2O3
 *   orc_zng_setup            mesh.F:2434-2512  NEleZNG, ZNGIF1-3 (IBTYPE 40)
 *   orc_mesh_neitabele       mesh.F:3110-3131, 3248-3283  NeiTabEle
 *   orc_coldstart_arrays     cstart.F:1332-1427 + totalAreaCalc mesh.F:3360-3400
 */
#include "oracle.h"

#include <cmath>
#include <vector>

namespace {
const double PI_ = 3.141592653589793;   /* constants.F90 PI */
const double RAD2DEG = 180.0 / PI_;     /* constants.F90 RAD2DEG */

/* 1-based column-major accessors for (rows, cols) Fortran arrays */
struct I2 {
  int *a;
  long rows;
  int &operator()(long i, long j) const { return a[(i - 1) + rows * (j - 1)]; }
};
struct CI2 {
  const int *a;
  long rows;
  int operator()(long i, long j) const { return a[(i - 1) + rows * (j - 1)]; }
};
}  // namespace

extern "C" {

/* mesh.F:1614-1664 (the ICS = 1 branch of the element loop): FDXE/FDYE
 * hold the shape-function derivative numerators, AREAS twice the signed
 * area; a clockwise element has NM(I,2) and NM(I,3) exchanged and is done
 * again (the reference's "reorder and start loop again").  Returns -1 for a
 * node number out of range, -2 for an element whose area stays <= 0. */
int orc_mesh_geometry(int np, int ne, const double *x, const double *y, int *nm,
                      double *fdxe, double *fdye, double *areas) {
  if (np <= 0 || ne <= 0) return -1;
  I2 NM{nm, ne};
  for (int i = 1; i <= ne; ++i) {
    for (int again = 0; again < 2; ++again) {
      const int n1 = NM(i, 1), n2 = NM(i, 2), n3 = NM(i, 3);
      if (n1 < 1 || n1 > np || n2 < 1 || n2 > np || n3 < 1 || n3 > np) return -1;
      const double X1 = x[n1 - 1], X2 = x[n2 - 1], X3 = x[n3 - 1];   /* EXV(1..3,I) */
      const double Y1 = y[n1 - 1], Y2 = y[n2 - 1], Y3 = y[n3 - 1];   /* EYV(1..3,I) */
      const double X2mX1 = (X2 - X1), X3mX2 = (X3 - X2), X1mX3 = (X1 - X3);
      const double Y2mY1 = (Y2 - Y1), Y3mY2 = (Y3 - Y2), Y1mY3 = (Y1 - Y3);
      double *fx = fdxe + 3L * (i - 1), *fy = fdye + 3L * (i - 1);
      fx[0] = -Y3mY2;
      fx[1] = -Y1mY3;
      fx[2] = -Y2mY1;
      fy[0] = X3mX2;
      fy[1] = X1mX3;
      fy[2] = X2mX1;
      areas[i - 1] = (X1mX3) * (-Y3mY2) + (X3mX2) * (Y1mY3);
      if (areas[i - 1] < 0.0 && again == 0) {
        const int t = NM(i, 2);
        NM(i, 2) = NM(i, 3);
        NM(i, 3) = t;
        continue;
      }
      break;
    }
    if (!(areas[i - 1] > 0.0)) return -2;
  }
  return 0;
}

/* mesh.F:1716-1731: NNeigh counts incident elements; MNEI = max + 2. */
int orc_mesh_mnei(int np, int ne, const int *nm) {
  CI2 NM{nm, ne};
  std::vector<int> nneigh(np + 1, 0);
  for (int i = 1; i <= ne; ++i)
    for (int k = 1; k <= 3; ++k) {
      const int n = NM(i, k);
      if (n < 1 || n > np) return -1;
      nneigh[n] = nneigh[n] + 1;
    }
  int mnei = 0;
  for (int n = 1; n <= np; ++n) mnei = std::max(mnei, nneigh[n]);
  return mnei + 2;
}

/* NEIGHB, mesh.F:3089-3318.  Edge pairs enter NeiTab in element order
 * (NN1-NN2, NN1-NN3, NN2-NN3), each neighbour remembering the element that
 * first contributed the edge (NeiTabETMP); then each node's neighbours are
 * sorted by increasing clockwise angle from east, measured with the element
 * vertex coordinates, and the node itself goes in slot 1.  Returns -3 when a
 * node has more than MNEI-1 neighbours (neighb_terminateDimensioning) and -4
 * for coincident nodes (neighb_terminateDuplicateNode). */
int orc_mesh_neighb(int np, int ne, int mnei, const double *x, const double *y, const int *nm,
                    int *nneigh, int *neitab, int *neimax) {
  CI2 NM{nm, ne};
  I2 NT{neitab, np};
  std::vector<int> etmp_v((size_t)np * mnei, 0);
  I2 ET{etmp_v.data(), np};
  for (int n = 1; n <= np; ++n) {
    nneigh[n - 1] = 0;
    for (int nn = 1; nn <= mnei; ++nn) NT(n, nn) = 0;
  }
  for (int n = 1; n <= ne; ++n) {
    const int nodes[3] = {NM(n, 1), NM(n, 2), NM(n, 3)};
    const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (const auto &pr : pairs) {
      const int a = nodes[pr[0]], b = nodes[pr[1]];
      bool found = false;
      for (int j = 1; j <= nneigh[a - 1]; ++j)
        if (b == NT(a, j)) {
          found = true;
          break;
        }
      if (!found) {
        nneigh[a - 1] = nneigh[a - 1] + 1;
        nneigh[b - 1] = nneigh[b - 1] + 1;
        if (nneigh[a - 1] > mnei - 1 || nneigh[b - 1] > mnei - 1) return -3;
        NT(a, nneigh[a - 1]) = b;
        NT(b, nneigh[b - 1]) = a;
        ET(a, nneigh[a - 1]) = n;
        ET(b, nneigh[b - 1]) = n;
      }
    }
  }
  std::vector<double> angle(mnei + 1, 0.0);
  std::vector<int> neitem(mnei + 1, 0);
  for (int i = 1; i <= np; ++i) {
    for (int j = 1; j <= nneigh[i - 1]; ++j) {
      neitem[j] = NT(i, j);
      /* DELX/DELY from the element vertex coordinates EXV/EYV of element EJ
         (mesh.F:3200-3211); ICS = 1 makes them X/Y of the two nodes */
      const int ej = ET(i, j);
      int ij = 0, ii = 0;
      for (int k = 1; k <= 3; ++k) {
        if (NM(ej, k) == neitem[j]) ij = k;
        if (NM(ej, k) == i) ii = k;
      }
      const double delx = x[NM(ej, ij) - 1] - x[NM(ej, ii) - 1];
      const double dely = y[NM(ej, ij) - 1] - y[NM(ej, ii) - 1];
      const double dist = std::sqrt(delx * delx + dely * dely);
      if (dist == 0.0) return -4;
      if (dely != 0.0) {
        angle[j] = RAD2DEG * std::acos(delx / dist);
        if (dely > 0.0) angle[j] = 360.0 - angle[j];
      }
      if (dely == 0.0) {
        if (delx > 0.0) angle[j] = 0.0;
        if (delx < 0.0) angle[j] = 180.0;
      }
    }
    double anglemore = -1.0;
    int jlow = 1;
    for (int jj = 1; jj <= nneigh[i - 1]; ++jj) {
      double anglelow = 400.0;
      for (int j = 1; j <= nneigh[i - 1]; ++j)
        if (angle[j] < anglelow && angle[j] > anglemore) {
          anglelow = angle[j];
          jlow = j;
        }
      NT(i, jj + 1) = neitem[jlow];
      anglemore = anglelow;
    }
    NT(i, 1) = i;
    nneigh[i - 1] = nneigh[i - 1] + 1;
  }
  int mx = 0;
  for (int n = 1; n <= np; ++n)
    if (nneigh[n - 1] > mx) mx = nneigh[n - 1];
  if (neimax) *neimax = mx;
  return 0;
}

/* compute_csr_positions, mesh.F:5261-5282: the NeiTab slot (2..NEIMAX) of
 * each of an element's two other nodes, per vertex.  Returns -1 if NEIMAX
 * exceeds MNEI and -5 if an element edge is missing from NeiTab (the
 * reference would leave the entry unset). */
int orc_mesh_csr_positions(int np, int ne, int mnei, const int *nm, const int *neitab, int neimax,
                           int *csr_position) {
  if (neimax > mnei) return -1;
  CI2 NM{nm, ne};
  CI2 NT{neitab, np};
  auto CP = [&](int i, int k, int l) -> int & {
    return csr_position[(i - 1) + (long)ne * ((k - 1) + 3L * (l - 1))];
  };
  for (int i = 1; i <= ne; ++i) {
    const int nn1 = NM(i, 1), nn2 = NM(i, 2), nn3 = NM(i, 3);
    for (int k = 1; k <= 3; ++k)
      for (int l = 1; l <= 2; ++l) CP(i, k, l) = 0;
    for (int jn = 2; jn <= neimax; ++jn) {
      if (NT(nn1, jn) == nn2) CP(i, 1, 1) = jn;
      if (NT(nn1, jn) == nn3) CP(i, 1, 2) = jn;
      if (NT(nn2, jn) == nn1) CP(i, 2, 1) = jn;
      if (NT(nn2, jn) == nn3) CP(i, 2, 2) = jn;
      if (NT(nn3, jn) == nn1) CP(i, 3, 1) = jn;
      if (NT(nn3, jn) == nn2) CP(i, 3, 2) = jn;
    }
    for (int k = 1; k <= 3; ++k)
      for (int l = 1; l <= 2; ++l)
        if (CP(i, k, l) == 0) return -5;
  }
  return 0;
}

/* Flow-boundary tables of mesh.F:2226-2568 for the land-segment types of
 * the path (external 0/10/20, island 1/11/21, specified flow 2/12/22,
 * radiation 30, coupled flux/radiation 32, zero normal gradient 40/41,
 * river radiation 52, external barrier 3/13/23, and each face of an
 * internal barrier 4/24 or 5/25 as its own unclosed segment, the back face reversed
 * as mesh.F:2158-2192 loads it):
 * segment closure (:2226-2244), per node the GWCE entry NBV/LBCODEI with
 * the inner-angle test (:2266-2411), BNDLEN2O3 (:2301-2303), the outward
 * normal CSII/SIII (:2421-2433, including the FLG_IBLEN2 special case of a
 * forced-closed two-node island), and the momentum key ME2GW (:2516-2568).
 * seg_ptr/seg_nodes list each segment's 1-based nodes as fort.14 does.
 * Returns -1 for an unsupported type, a segment shorter than 2 or a node out
 * of range, -6 when more than nvel_max entries are needed. */
int orc_boundary_setup(int np, const double *x, const double *y, int nbou, const int *ibtype,
                       const int *seg_ptr, const int *seg_nodes, double costset, int nvel_max,
                       int *nvel_out, int *nbv, int *lbcodei, double *csii, double *siii,
                       int *nvelme_out, int *me2gw, double *bndlen2o3) {
  auto flow_first = [](int c) {   /* codes the momentum equation keeps at an overlap */
    return c == 2 || c == 12 || c == 22 || c == 3 || c == 13 || c == 23 || c == 30 ||
           c == 32 || c == 40 || c == 41 || c == 52 || c == 64;
  };
  int jgw = 0, jme = 0;
  for (int k = 0; k < nbou; ++k) {
    const int t = ibtype[k];
    const bool island = (t == 1 || t == 11 || t == 21);
    if (!(island || t == 0 || t == 10 || t == 20 || t == 2 || t == 12 || t == 22 || t == 30 ||
          t == 32 || t == 40 || t == 41 || t == 52 || t == 3 || t == 13 || t == 23 || t == 4 ||
          t == 24 || t == 5 || t == 25))
      return -1;
    int nvell = seg_ptr[k + 1] - seg_ptr[k];
    if (nvell < 2) return -1;
    std::vector<int> nbvv(nvell + 3, 0);   /* NBVV(K,0:NVELL+1) */
    for (int i = 1; i <= nvell; ++i) {
      nbvv[i] = seg_nodes[seg_ptr[k] + i - 1];
      if (nbvv[i] < 1 || nbvv[i] > np) return -1;
    }
    bool flg_iblen2 = false;
    nbvv[0] = nbvv[1];                                   /* unclosed external */
    if (island && nbvv[nvell] != nbvv[1]) {             /* close an unclosed internal */
      if (nvell == 2) flg_iblen2 = true;
      nvell = nvell + 1;
      nbvv.resize(nvell + 3, 0);
      nbvv[nvell] = nbvv[1];
    }
    if (nbvv[nvell] == nbvv[1]) nbvv[0] = nbvv[nvell - 1];   /* closed */
    nbvv[nvell + 1] = nbvv[nvell];
    double theta1 = 0.0, cross1 = 0.0, costheta1 = 0.0;
    for (int i = 1; i <= nvell; ++i) {
      jgw = jgw + 1;
      if (jgw > nvel_max) return -6;
      const int nbvi = nbvv[i], nbvj = nbvv[i + 1], nbvk = nbvv[i - 1];
      nbv[jgw - 1] = nbvi;
      double xgj = x[nbvj - 1], ygj = y[nbvj - 1];
      const double xgi = x[nbvi - 1], ygi = y[nbvi - 1];
      const double xgk = x[nbvk - 1], ygk = y[nbvk - 1];
      const double delx = xgj - xgi, dely = ygj - ygi;
      bndlen2o3[jgw - 1] = 2.0 * (std::sqrt(delx * delx + dely * dely)) / 3.0;
      double theta = 0.0, cross = 0.0, costheta = 0.0;
      bool calc_theta = true;
      if (i == 1 && nbvv[1] == nbvv[0]) {
        theta = -9999999.0;
        cross = 0.0;
        costheta = costset;
        calc_theta = false;
      }
      if (i == nvell) {
        theta = theta1;
        cross = cross1;
        costheta = costheta1;
        calc_theta = false;
      }
      if (calc_theta) {
        const double vl1x = xgk - xgi, vl1y = ygk - ygi;
        const double vl2x = xgj - xgi, vl2y = ygj - ygi;
        const double dotvec = vl1x * vl2x + vl1y * vl2y;
        const double vecnorm =
            (std::sqrt(vl1x * vl1x + vl1y * vl1y)) * (std::sqrt(vl2x * vl2x + vl2y * vl2y));
        costheta = dotvec / vecnorm;
        if (costheta > 1.0) costheta = 1.0;
        if (costheta < -1.0) costheta = -1.0;
        theta = RAD2DEG * std::acos(costheta);
        cross = -vl1x * vl2y + vl2x * vl1y;
        if (cross < 0) theta = 360.0 - theta;
      }
      if (i == 1) {
        theta1 = theta;
        cross1 = cross;
        costheta1 = costheta;
      }
      (void)theta;
      lbcodei[jgw - 1] = t;
      if (costheta > costset && cross > 0.0) {   /* 2DDI: zero tangential slip */
        if (t == 0) lbcodei[jgw - 1] = 10;
        if (t == 1) lbcodei[jgw - 1] = 11;
        if (t == 2) lbcodei[jgw - 1] = 12;
        if (t == 3) lbcodei[jgw - 1] = 13;
      }
      if (flg_iblen2) {
        xgj = xgi;
        ygj = ygi;
      }
      const double xl = std::sqrt((xgk - xgj) * (xgk - xgj) + (ygk - ygj) * (ygk - ygj));
      csii[jgw - 1] = 1.0 * (ygj - ygk) / xl;   /* SFMX = 1 */
      siii[jgw - 1] = (xgk - xgj) / xl;
      if (i == 1) {
        if (jgw == 1) {
          jme = jme + 1;
          me2gw[jme - 1] = jgw;
        }
        if (jgw != 1) {
          if (nbv[jgw - 1] != nbv[jgw - 2]) {
            jme = jme + 1;
            me2gw[jme - 1] = jgw;
          }
          if (nbv[jgw - 1] == nbv[jgw - 2] && flow_first(lbcodei[jgw - 1])) me2gw[jme - 1] = jgw;
        }
      }
      if (i > 1 && i < nvell) {
        jme = jme + 1;
        me2gw[jme - 1] = jgw;
      }
      if (i == nvell) {
        if (nbv[jgw - 1] != nbvv[1] && nbv[jgw - 1] != nbv[0]) {
          jme = jme + 1;
          me2gw[jme - 1] = jgw;
        }
        if (nbvv[i] == nbv[0] && flow_first(lbcodei[jgw - 1])) me2gw[0] = jgw;
      }
    }
  }
  *nvel_out = jgw;
  *nvelme_out = jme;
  return 0;
}

/* NeiTabEle, NEIGHB mesh.F:3110-3131 (each element appended to its three
 * nodes' lists in element order) and :3248-3283 (for J = 2..NNeigh, the
 * element (NN1, NN2, NN3) = (I, NeiTab(I,J+1) or NeiTab(I,2) at the end,
 * NeiTab(I,J)) in counter-clockwise order, packed as NN = NN + 1). */
int orc_mesh_neitabele(int np, int ne, int mnei, const int *nm, const int *nneigh,
                       const int *neitab, int *neitabele) {
  if (np <= 0 || ne <= 0 || mnei < 3) return -1;
  CI2 NM{nm, ne}, NeiTab{neitab, np};
  I2 NeiTabEle{neitabele, np};
  std::vector<int> NNeighEle(np + 1, 0);
  std::vector<int> lists((size_t)np * mnei * 2, 0);   /* elements around each node */
  const int cap = mnei * 2;
  for (int i = 1; i <= np; ++i)
    for (int k = 1; k <= mnei; ++k) NeiTabEle(i, k) = 0;
  for (int N = 1; N <= ne; ++N)
    for (int k = 1; k <= 3; ++k) {
      const int v = NM(N, k);
      if (v < 1 || v > np || NNeighEle[v] >= cap) return -1;
      lists[(size_t)(v - 1) * cap + NNeighEle[v]] = N;
      NNeighEle[v] = NNeighEle[v] + 1;
    }
  for (int I = 1; I <= np; ++I) {
    std::vector<int> NEITEM(lists.begin() + (size_t)(I - 1) * cap,
                            lists.begin() + (size_t)(I - 1) * cap + NNeighEle[I]);
    int NN = 0;
    for (int J = 2; J <= nneigh[I - 1]; ++J) {
      const int NN1 = NeiTab(I, 1);
      const int NN3 = NeiTab(I, J);
      const int NN2 = J != nneigh[I - 1] ? NeiTab(I, J + 1) : NeiTab(I, 2);
      int NE1 = 0, NE2 = 0, NE3 = 0;
      for (int K = 0; K < (int)NEITEM.size(); ++K) {
        if (NEITEM[K] == 0) continue;
        const int e = NEITEM[K];
        if (NM(e, 1) == NN1) { NE1 = NM(e, 1); NE2 = NM(e, 2); NE3 = NM(e, 3); }
        if (NM(e, 2) == NN1) { NE1 = NM(e, 2); NE2 = NM(e, 3); NE3 = NM(e, 1); }
        if (NM(e, 3) == NN1) { NE1 = NM(e, 3); NE2 = NM(e, 1); NE3 = NM(e, 2); }
        if (NE2 == NN2 && NE3 == NN3) {
          NN = NN + 1;
          if (NN > mnei) return -1;
          NeiTabEle(I, NN) = e;
          NEITEM[K] = 0;
          break;
        }
      }
      (void)NE1;
    }
  }
  return 0;
}

/* Zero-normal-gradient fictitious nodes, mesh.F:2434-2512: for each
 * IBTYPE 40 entry JGW, ZNGFicNodeDist = 1.001 x the largest distance to the
 * NeiTab neighbours, X4/Y4 that far inward along -(CSII, SIII), NEleZNG the
 * element minimising |AA - AREAS|/AREAS (strict <, so the first one wins)
 * and ZNGIF1-3 the interpolation factors. */
int orc_zng_setup(int np, int ne, const double *x, const double *y, const int *nm, int mnei,
                  const int *nneigh, const int *neitab, const double *areas, int nvel,
                  const int *nbv, const int *lbcodei, const double *csii, const double *siii,
                  int *nelezng, double *zngif1, double *zngif2, double *zngif3) {
  if (np <= 0 || ne <= 0 || nvel < 0) return -1;
  CI2 NM{nm, ne}, NeiTab{neitab, np};
  auto X = [&](int n) { return x[n - 1]; };
  auto Y = [&](int n) { return y[n - 1]; };
  for (int JGW = 1; JGW <= nvel; ++JGW) {
    nelezng[JGW - 1] = 0;
    zngif1[JGW - 1] = zngif2[JGW - 1] = zngif3[JGW - 1] = 0.0;
    if (lbcodei[JGW - 1] != 40) continue;
    const int NBVI = nbv[JGW - 1];
    if (NBVI < 1 || NBVI > np) return -1;
    double ZNGFicNodeDist = 0.0;
    for (int N = 2; N <= nneigh[NBVI - 1] && N <= mnei; ++N) {
      const int nb = NeiTab(NBVI, N);
      if (nb < 1 || nb > np) return -1;
      const double ZNGFicNodeDistTemp = std::sqrt((X(nb) - X(NBVI)) * (X(nb) - X(NBVI)) +
                                                  (Y(nb) - Y(NBVI)) * (Y(nb) - Y(NBVI)));
      if (ZNGFicNodeDist < ZNGFicNodeDistTemp) ZNGFicNodeDist = ZNGFicNodeDistTemp;
    }
    ZNGFicNodeDist = 1.001 * ZNGFicNodeDist;
    const double X4 = X(NBVI) - ZNGFicNodeDist * csii[JGW - 1];
    const double Y4 = Y(NBVI) - ZNGFicNodeDist * siii[JGW - 1];
    double AEMIN = (double)1.0E+25f;
    int NEle = 0;
    for (int N = 1; N <= ne; ++N) {
      const int N1 = NM(N, 1), N2 = NM(N, 2), N3 = NM(N, 3);
      const double X1 = X(N1), X2 = X(N2), X3 = X(N3), Y1 = Y(N1), Y2 = Y(N2), Y3 = Y(N3);
      const double A1 = (X4 - X3) * (Y2 - Y3) + (X2 - X3) * (Y3 - Y4);
      const double A2 = (X4 - X1) * (Y3 - Y1) - (Y4 - Y1) * (X3 - X1);
      const double A3 = (Y4 - Y1) * (X2 - X1) - (X4 - X1) * (Y2 - Y1);
      const double AA = std::fabs(A1) + std::fabs(A2) + std::fabs(A3);
      const double AE = std::fabs(AA - areas[N - 1]) / areas[N - 1];
      if (AE < AEMIN) {
        AEMIN = AE;
        NEle = N;
      }
    }
    if (NEle == 0) return -1;
    const int N1 = NM(NEle, 1), N2 = NM(NEle, 2), N3 = NM(NEle, 3);
    const double X1 = X(N1), X2 = X(N2), X3 = X(N3), Y1 = Y(N1), Y2 = Y(N2), Y3 = Y(N3);
    nelezng[JGW - 1] = NEle;
    zngif1[JGW - 1] = ((X4 - X3) * (Y2 - Y3) + (X2 - X3) * (Y3 - Y4)) / areas[NEle - 1];
    zngif2[JGW - 1] = ((X4 - X1) * (Y3 - Y1) - (Y4 - Y1) * (X3 - X1)) / areas[NEle - 1];
    zngif3[JGW - 1] = (-(X4 - X1) * (Y2 - Y1) + (Y4 - Y1) * (X2 - X1)) / areas[NEle - 1];
  }
  return 0;
}

/* Cold start with the library's argument list: fills the structs the
 * oracle's orc_coldstart (cstart.F:1332-1427, totalAreaCalc mesh.F:
 * 3360-3400) reads. */
int orc_coldstart_arrays(int np, int ne, int nolifa, double h0, const double *dp, const int *nm,
                         const double *areas, double *eta1, double *eta2, int *nnodecode,
                         int *nodecode, int *noff, int *mju, double *totalarea) {
  if (np <= 0 || ne <= 0) return -1;
  orc_params_t p{};
  p.nolifa = nolifa;
  p.h0 = h0;
  orc_arrays_t a{};
  a.np = np;
  a.ne = ne;
  a.dp = dp;
  a.nm = nm;
  a.areas = areas;
  a.eta1 = eta1;
  a.eta2 = eta2;
  a.nnodecode = nnodecode;
  a.nodecode = nodecode;
  a.noff = noff;
  a.mju = mju;
  a.totalarea = totalarea;
  orc_coldstart(&p, &a);
  return 0;
}

}  /* extern "C" */
