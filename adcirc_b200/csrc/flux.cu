// flux.cu -- specified normal flux boundaries (IBTYPE 2, 12, 22), external
// barriers (3, 13, 23), internal barriers (4, 24) and barriers with pipes
// (5, 25), radiation boundaries (30), coupled flux/radiation boundaries
// (32), zero-normal-gradient boundaries (40, 41) and river-radiation
// boundaries (52).
//
// Three pieces of the reference's flux-boundary path:
//  * QN0 <- QN1 <- QN2 <- 0 and EN0 <- EN1 <- EN2 <- 0 (timestep.F:606-613),
//    then QN2 (and at IBTYPE 32 entries EN2) as the sum of the periodic
//    constituents (timestep.F:861-880; ICS = 1, so the normal flux is not
//    rotated), and at radiation entries QN1 = H2 (UU1 CSII +
//    VV1 SIII), the discharge of the latest velocity (timestep.F:932-940),
//    and the same at zero-normal-gradient entries (:945-952);
//    river-radiation entries take their discharge elevation ElevDisc at
//    FluxSettlingIT (or from the cold-start EtaDisc, timestep.F:906-926);
//  * the GWCE boundary line integral (gwce.F:1737-1834): a force per
//    boundary entry (specified flux, the radiation condition
//    -sqrt(g H1) ETAS / DT - TAU0 QN1, the coupled condition of IBTYPE 32
//    against the specified elevation EN, or for river radiation the specified
//    flux less sqrt(g H1) (ETAS / DT + TAU0 (ETA1 - ElevDisc)) after
//    FluxSettlingIT), then for each pair of consecutive
//    entries a contribution to both nodes.  The reference adds these in entry order;
//    here one thread per boundary node adds its contributions in that same
//    order (a table built at bind lists them), so GWCE_LV gets the same bits;
//  * the specified normal velocity -QN2/H2 of the momentum boundary
//    conditions (momentum.F:815-856), read in k_mom_node; radiation nodes
//    take no momentum boundary condition.
// External barriers (IBTYPE 3/13/23) take as QN2 the free-surface
// supercritical outflow over the crest once the water stands BARMIN above it
// (COMPUTE_EXTERNAL_BOUNDARY_FLUX, weir_boundary.F90:1727-1763, called from
// timestep.F:967-975 after the other fluxes); the GWCE integral and the
// momentum equations then treat them like specified-flux entries.
// Internal barriers (IBTYPE 4/24) pass water between the paired nodes of
// their two faces (COMPUTE_INTERNAL_BOUNDARY_FLUX, weir_boundary.F90:
// 1775-1942, called per entry from timestep.F:1003-1026): sub- or
// supercritical weir flow from the higher side once it stands BARMIN over
// the crest, none while the source node or all its neighbours along the
// barrier are dry; a receiving node is flagged in NIBNODECODE, which the
// wet/dry step uses (wetdry.F:813-816, 1086-1090, 1114).  Barriers with
// pipes (IBTYPE 5/25) add the free or submerged discharge through the pipe
// under the crown (COMPUTE_CROSS_BARRIER_PIPE_FLUX, weir_boundary.F90:
// 2469-2579, timestep.F:1034-1044).
// It also holds the non-periodic boundary series: fort.20 fluxes in place of
// the periodic constituents (NFFR <= 0, timestep.F:882-903) and fort.19
// elevations added to the periodic boundary elevation in k_eta_bc
// (gwce.F:1659-1674).  Both files sit whole in HBM; k_series_state moves
// the pair of record times as the reference's reads do.
#include "adc_internal.cuh"

#include <cmath>
#include <cstring>
#include <vector>

namespace adc {

// One thread: per active series, the record pair and ratio of this step.
// The reference reads the next record when TimeLoc passes the later record
// time, at most once per step (gwce.F:1660-1668, timestep.F:882-900).
__global__ void k_series_state(adc_ctx c, const adc_step_t *steps, Flags *flags) {
  griddep_wait();
  const double timeloc = steps[flags->cursor].timeloc;
  for (int s = 0; s < 2; ++s) {
    if (!(s == 0 ? c.eser_on : c.fser_on)) continue;
    SeriesState &st = c.sstate[s];
    const int nrec = s == 0 ? c.eser_nrec : c.fser_nrec;
    const double inc = s == 0 ? c.eser_interval : c.fser_interval;
    if (timeloc > st.t2) {
      st.t1 = st.t2;
      st.t2 = st.t1 + inc;
      st.k = st.k + 1;
      if (st.k + 1 >= nrec) {   // the file has no further record
        st.err = 1;
        flags->status = ADC_ERR_ARG;
        st.k = nrec - 2;
      }
    }
    st.ratio = (timeloc - st.t1) / inc;
  }
}

// COMPUTE_INTERNAL_BOUNDARY_FLUX (weir_boundary.F90:1775-1942, the default
// wet-edge formulation without averaging); the square roots stand for the
// reference's **0.5.
__device__ double internal_barrier_flux(const adc_ctx &c, int I, double ramp) {
  const int n1 = c.bnv[I], n2 = c.ibconn[I], kind = c.ibkind[I];
  const int *nc = c.nodecode;
  int wn1 = 0, wn2 = 0;   // wet neighbours along the barrier on each side
  if (kind == 0) {
    wn1 = wn1 + nc[c.bnv[I + 1]];
    wn2 = wn2 + nc[c.ibconn[I + 1]];
  } else if (kind == 1) {
    wn1 = wn1 + nc[c.bnv[I - 1]];
    wn2 = wn2 + nc[c.ibconn[I - 1]];
  } else {
    wn1 = wn1 + nc[c.bnv[I - 1]];
    wn1 = wn1 + nc[c.bnv[I + 1]];
    wn2 = wn2 + nc[c.ibconn[I + 1]];
    wn2 = wn2 + nc[c.ibconn[I - 1]];
  }
  const double R1 = c.eta2[n1] - c.binht[I], R2 = c.eta2[n2] - c.binht[I];
  const double R1F = 2.0 * R1 / 3.0, R2F = 2.0 * R2 / 3.0;
  const double G = c.p.g, BARMIN = 0.04;
  double flux = 0.0;
  if ((R1 < 0.0) && (R2 < 0.0)) {
    flux = 0.0;
  } else if (fabs(R1 - R2) < 0.01) {
    flux = 0.0;
  } else if ((R1 > R2) && (R1 > BARMIN)) {   // this side is the source
    if (nc[n1] == 0 || wn1 == 0) flux = 0.0;
    else if (R2 > R1F) flux = -ramp * R2 * c.bincfsb[I] * sqrt(2.0 * G * (R1 - R2));
    else flux = -ramp * c.bincfsp[I] * R1F * sqrt(R1F * G);
  } else if ((R2 > R1) && (R2 > BARMIN)) {   // this side receives
    if (nc[n2] == 0 || wn2 == 0) {
      flux = 0.0;
    } else {
      if (R1 > R2F) flux = ramp * R1 * c.bincfsb[I] * sqrt(2.0 * G * (R2 - R1));
      else flux = ramp * c.bincfsp[I] * R2F * sqrt(R2F * G);
      c.nib[n1] = 1;
    }
  }
  return flux;
}

// COMPUTE_CROSS_BARRIER_PIPE_FLUX (weir_boundary.F90:2469-2579); the
// reference's **0.5 as square roots and PIPEDIAM**2 as a product.
__device__ double pipe_flux(const adc_ctx &c, int I, double ramp) {
  const int n1 = c.bnv[I], n2 = c.ibconn[I];
  const double *pp = c.pipe;
  const double ht = pp[I], coef = pp[c.nvel + I], diam = pp[2 * c.nvel + I];
  const double G = c.p.g, BARMIN = 0.04, PI = 3.141592653589793;
  const double R1 = c.eta2[n1] - ht, R2 = c.eta2[n2] - ht;
  if ((R1 < 0.0) && (R2 < 0.0)) return 0.0;
  if (fabs(R1 - R2) < BARMIN) return 0.0;
  double flux = 0.0;
  if ((R1 > R2) && (R1 > BARMIN)) {   // outward
    if (R2 <= 0.0) {
      flux = c.nodecode[n1] == 0 ? 0.0
                                 : -ramp * 0.25 * PI * (diam * diam) * sqrt(2.0 * G * R1 / (1.0 + coef));
    } else {
      return c.nodecode[n1] == 0 ? 0.0
                                 : -ramp * 0.25 * PI * (diam * diam) * sqrt(2.0 * G * (R1 - R2) / coef);
    }
  }
  if ((R2 > R1) && (R2 > BARMIN)) {   // inward
    if (c.nodecode[n2] == 0) return 0.0;
    if (R1 <= 0.0) flux = ramp * 0.25 * PI * (diam * diam) * sqrt(2.0 * G * R2 / (1.0 + coef));
    else flux = ramp * 0.25 * PI * (diam * diam) * sqrt(2.0 * G * (R2 - R1) / coef);
    c.nib[n1] = 1;
  }
  return flux;
}

__global__ void k_flux_forcing(adc_ctx c, const adc_step_t *steps, const Flags *flags) {
  griddep_wait();
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= c.nvel) return;
  double *qn0 = c.qn, *qn1 = c.qn + c.nvel, *qn2 = c.qn + 2 * c.nvel;
  double *en0 = c.en, *en1 = c.en + c.nvel, *en2 = c.en + 2 * c.nvel;
  qn0[I] = qn1[I];
  qn1[I] = qn2[I];
  en0[I] = en1[I];
  en1[I] = en2[I];
  double q = 0.0, el = 0.0;
  const int lb = c.blbc[I];
  const adc_step_t st = steps[flags->cursor];
  if (c.flux_on && (lb == 2 || lb == 12 || lb == 22 || lb == 32 || lb == 52)) {
    const int nf = c.nffr;
    const size_t nfv = (size_t)nf * c.nvel;
    const double *famig = c.fconst, *fper = famig + nf, *fff = fper + nf, *fface = fff + nf;
    const double *qnam = c.fqn, *qnph = c.fqn + nfv, *enam = qnph + nfv, *enph = enam + nfv;
    const bool coupled = lb == 32 && c.fen;
    for (int J = 0; J < nf; ++J) {
      int NCYC = 0;
      if (fper[J] != 0.0) NCYC = (int)(st.timeh / fper[J]);
      const double ARGJ = famig[J] * (st.timeh - NCYC * fper[J]) + fface[J];
      const double RFF = fff[J] * st.rampextflux;
      q = q + qnam[J + (size_t)nf * I] * RFF * cos(ARGJ - qnph[J + (size_t)nf * I]);
      if (coupled) el = el + enam[J + (size_t)nf * I] * RFF * cos(ARGJ - enph[J + (size_t)nf * I]);
    }
  } else if (c.fser_on) {   // timestep.F:900-902, every entry
    const SeriesState &ss = c.sstate[1];
    const size_t r1 = (size_t)ss.k * c.nvel, r2 = r1 + c.nvel;
    q = st.rampextflux * (c.fser_q[r1 + I] + ss.ratio * (c.fser_q[r2 + I] - c.fser_q[r1 + I]));
    el = st.rampextflux * (c.fser_e[r1 + I] + ss.ratio * (c.fser_e[r2 + I] - c.fser_e[r1 + I]));
  }
  if (lb == 3 || lb == 13 || lb == 23) {
    // the weir formula with g and BARMIN = 0.04 m (weir_boundary.F90:51);
    // (RBARWL g)^0.5 as a square root
    const double RBARWL = 2.0 * (c.eta2[c.bnv[I]] - c.barht[I]) / 3.0;
    q = RBARWL > 0.04 ? -st.rampintflux * c.barcf[I] * RBARWL * sqrt(RBARWL * c.p.g) : 0.0;
  }
  if (lb == 4 || lb == 24 || lb == 5 || lb == 25) q = internal_barrier_flux(c, I, st.rampintflux);
  if (lb == 5 || lb == 25) q = q + pipe_flux(c, I, st.rampintflux);   // timestep.F:1034-1044
  qn2[I] = q;
  en2[I] = el;
  if (lb == 52) {
    const int n = c.bnv[I];
    if (st.it == c.flux_settling_it) {
      c.etadisc_b[I] = c.eta2[n];
      c.elevdisc[I] = c.eta2[n];
    } else if (!flags->etadisc_done && st.it > c.flux_settling_it) {
      c.elevdisc[I] = c.etadisc_b[I];
    }
  }
  if (lb == 30 || lb == 40 || lb == 41) {
    const int n = c.bnv[I];
    const double UN1 = c.uu1[n] * c.bcsii[I] + c.vv1[n] * c.bsiii[I];
    qn1[I] = c.h2[n] * UN1;
  }
}

// The force of each boundary entry (gwce.F:1783-1815): LBCODEI <= 29 from
// the specified flux, 30 the radiation condition with the saved H1, 52 the
// specified flux plus, after FluxSettlingIT, the radiation term.
__global__ void k_flux_qforce(adc_ctx c, const adc_step_t *steps, Flags *flags) {
  griddep_wait();
  const int J = blockIdx.x * blockDim.x + threadIdx.x;
  const int it = steps[flags->cursor].it;
  // EtaDisc_Fill ends with the first step at or after FluxSettlingIT; the
  // forcing kernel of this step has read it already
  if (J == 0 && it >= c.flux_settling_it) flags->etadisc_done = 1;
  if (J >= c.nvel) return;
  const double *qn0 = c.qn, *qn1 = c.qn + c.nvel, *qn2 = c.qn + 2 * c.nvel;
  const int n = c.bnv[J];
  if (c.blbc[J] == 32) {   // gwce.F:1792-1797
    const double *en0 = c.en, *en1 = c.en + c.nvel, *en2 = c.en + 2 * c.nvel;
    const double CELERITY = sqrt(c.p.g * c.h1[n]);
    const double DT2 = c.p.dt * 2.0;
    c.qforce[J] = (qn2[J] - qn0[J]) / DT2 - CELERITY * (2.0 * c.etas[n] - (en2[J] - en0[J])) / DT2 +
                  c.tau0[n] * (qn1[J] - CELERITY * (c.eta1[n] - en1[J]));
    return;
  }
  if (c.blbc[J] == 40 || c.blbc[J] == 41) {   // gwce.F:1804-1805
    c.qforce[J] = -(qn1[J] - qn0[J]) / c.p.dt - c.tau0[n] * (qn1[J] + qn0[J]) / 2.0;
    return;
  }
  if (c.blbc[J] == 30) {
    const double CELERITY = sqrt(c.p.g * c.h1[n]);
    c.qforce[J] = -CELERITY * c.etas[n] / c.p.dt - c.tau0[n] * qn1[J];
    return;
  }
  const double DT2 = c.p.dt * 2.0;
  double q = (qn2[J] - qn0[J]) / DT2 + c.tau0[n] * qn1[J];
  if (c.blbc[J] == 52 && it > c.flux_settling_it) {
    const double Celerity = sqrt(c.p.g * c.h1[n]);
    q = q - Celerity * (c.etas[n] / c.p.dt + c.tau0[n] * (c.eta1[n] - c.elevdisc[J]));
  }
  c.qforce[J] = q;
}

// One thread per boundary node: its contributions in entry order.
__global__ void k_flux_rhs(adc_ctx c) {
  griddep_wait();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.n_fx) return;
  const int n = c.fx_node[k];
  double v = c.gwce_lv[n];
  for (int q = c.fx_ptr[k]; q < c.fx_ptr[k + 1]; ++q) {
    const int ent = c.fx_ent[q], j = ent >> 1;
    const int NCI = c.nodecode[c.bnv[j - 1]], NCJ = c.nodecode[c.bnv[j]];
    const double B = NCI * NCJ * c.bbl[j - 1] / 4.0;
    const double qi = c.qforce[j - 1], qj = c.qforce[j];
    if ((ent & 1) == 0) v = v + B * (2.0 * qi + qj);   // the segment's first node
    else v = v + B * (2.0 * qj + qi);                  // its second node
  }
  c.gwce_lv[n] = v;
}

int launch_flux_forcing(adc_ctx *c) {
  if (c->eser_on || c->fser_on) {
    launch_k(k_series_state, 1, 1, c->stream, *c, c->steps, c->flags);
    c->launches++;
  }
  if (!c->nfluxf && !c->nfluxrbc && !c->nfluxgbc && !c->nfluxb && !c->nfluxib) return ADC_OK;
  launch_k(k_flux_forcing, nblk(c->nvel), kThreads, c->stream, *c, c->steps, c->flags);
  c->launches++;
  return ADC_OK;
}

int launch_flux_rhs(adc_ctx *c) {
  if (!c->nfluxf && !c->nfluxrbc && !c->nfluxgbc && !c->nfluxb && !c->nfluxib) return ADC_OK;
  launch_k(k_flux_qforce, nblk(c->nvel), kThreads, c->stream, *c, c->steps, c->flags);
  launch_k(k_flux_rhs, nblk(c->n_fx), kThreads, c->stream, *c);
  c->launches += 2;
  return ADC_OK;
}

// Bind-time tables: boundary entries, and per boundary node the ordered
// list of (segment, side) contributions of the GWCE line integral.
int flux_tables(adc_ctx *c, const adc_arrays_t *a) {
  const int nv = a->nvel;
  c->nvel = nv;
  c->nfluxf = 0;
  c->nfluxrbc = 0;
  c->nfluxgbc = 0;
  c->nfluxb = 0;
  c->nfluxib = 0;
  c->nfluxibp = 0;
  for (int I = 0; I < nv; ++I) {
    const int lb = a->lbcodei[I];
    if (lb == 3 || lb == 13 || lb == 23) c->nfluxb = 1;
    if (lb == 4 || lb == 24 || lb == 5 || lb == 25) c->nfluxib = 1;
    if (lb == 5 || lb == 25) c->nfluxibp = 1;
    if (lb == 2 || lb == 12 || lb == 22 || lb == 32 || lb == 52) c->nfluxf = 1;
    if (lb == 30 || lb == 32) c->nfluxrbc = 1;
    if (lb == 40 || lb == 41) c->nfluxgbc = 1;
    if (lb == 64) {
      set_error("boundary code %d (condensed nodes) is not implemented", lb);
      return ADC_ERR_UNSUPPORTED;
    }
  }
  const size_t nva = (size_t)(nv > 0 ? nv : 1);
  ADC_CUDA(cudaMalloc((void **)&c->qn, 3 * nva * sizeof(double)));
  ADC_CUDA(cudaMemset(c->qn, 0, 3 * nva * sizeof(double)));
  ADC_CUDA(cudaMalloc((void **)&c->en, 3 * nva * sizeof(double)));
  ADC_CUDA(cudaMemset(c->en, 0, 3 * nva * sizeof(double)));
  if (!c->nfluxf && !c->nfluxrbc && !c->nfluxgbc && !c->nfluxb && !c->nfluxib) return ADC_OK;
  if (c->nfluxb && (!a->barlanht || !a->barlancfsp)) {
    set_error("the mesh has external barriers (IBTYPE 3/13/23) but no BARLANHT/BARLANCFSP");
    return ADC_ERR_MESH;
  }
  std::vector<int> bnv(nv);
  for (int I = 0; I < nv; ++I) bnv[I] = a->nbv[I] - 1;
  std::vector<std::vector<int>> lists(c->np);
  std::vector<int> order;
  auto add = [&](int node, int ent) {
    if (lists[node].empty()) order.push_back(node);
    lists[node].push_back(ent);
  };
  for (int j = 1; j < nv; ++j) {
    add(bnv[j - 1], j << 1);
    add(bnv[j], (j << 1) | 1);
  }
  std::vector<int> ptr(1, 0), ent;
  for (int n : order) {
    ent.insert(ent.end(), lists[n].begin(), lists[n].end());
    ptr.push_back((int)ent.size());
  }
  c->n_fx = (int)order.size();
  auto up_i = [&](int **d, const std::vector<int> &h) -> int {
    ADC_CUDA(cudaMalloc((void **)d, std::max<size_t>(h.size(), 1) * sizeof(int)));
    if (!h.empty()) ADC_CUDA(cudaMemcpy(*d, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice));
    return ADC_OK;
  };
  int rc;
  if ((rc = up_i(&c->bnv, bnv))) return rc;
  if ((rc = up_i(&c->blbc, std::vector<int>(a->lbcodei, a->lbcodei + nv)))) return rc;
  if ((rc = up_i(&c->fx_node, order))) return rc;
  if ((rc = up_i(&c->fx_ptr, ptr))) return rc;
  if ((rc = up_i(&c->fx_ent, ent))) return rc;
  ADC_CUDA(cudaMalloc((void **)&c->bbl, nva * sizeof(double)));
  ADC_CUDA(cudaMemcpy(c->bbl, a->bndlen2o3, nv * sizeof(double), cudaMemcpyHostToDevice));
  ADC_CUDA(cudaMalloc((void **)&c->qforce, nva * sizeof(double)));
  ADC_CUDA(cudaMalloc((void **)&c->bcsii, nva * sizeof(double)));
  ADC_CUDA(cudaMalloc((void **)&c->bsiii, nva * sizeof(double)));
  ADC_CUDA(cudaMemcpy(c->bcsii, a->csii, nv * sizeof(double), cudaMemcpyHostToDevice));
  ADC_CUDA(cudaMemcpy(c->bsiii, a->siii, nv * sizeof(double), cudaMemcpyHostToDevice));
  // internal barriers: the entry's place on its face, as the loop of
  // timestep.F:1003-1026 walks the segments (J = 1..2 NVELL per barrier)
  std::vector<int> ibk(nva, -1), ibc(nva, 0);
  if (c->nfluxib) {
    if (!a->ibconn || !a->barinht || !a->barincfsb || !a->barincfsp || !a->nvell || a->nbou < 1) {
      set_error("the mesh has internal barriers (IBTYPE 4/24) but no IBCONN/BARINHT/BARINCFSB/"
                "BARINCFSP/NVELL");
      return ADC_ERR_MESH;
    }
    int I = 0;
    for (int K = 0; K < a->nbou; ++K) {
      if (I >= nv) {
        set_error("NVELL overruns NVEL at boundary segment %d", K + 1);
        return ADC_ERR_MESH;
      }
      const int lb = a->lbcodei[I], n = a->nvell[K];
      if (lb == 4 || lb == 24 || lb == 5 || lb == 25) {
        if (I + 2 * n > nv || n < 2) {
          set_error("internal barrier segment %d does not fit NVEL", K + 1);
          return ADC_ERR_MESH;
        }
        for (int J = 1; J <= 2 * n; ++J, ++I) {
          ibk[I] = (J == 1 || J == n + 1) ? 0 : (J == n || J == 2 * n) ? 1 : 2;
          const int across = a->ibconn[I];
          if (across < 1 || across > c->np) {
            set_error("IBCONN of boundary entry %d is out of range", I + 1);
            return ADC_ERR_MESH;
          }
          ibc[I] = across - 1;
        }
      } else {
        I += n;
      }
    }
    if (I != nv) {
      set_error("NVELL adds up to %d boundary entries, NVEL is %d", I, nv);
      return ADC_ERR_MESH;
    }
  }
  if ((rc = up_i(&c->ibkind, ibk))) return rc;
  if ((rc = up_i(&c->ibconn, ibc))) return rc;
  for (double **d : {&c->binht, &c->bincfsb, &c->bincfsp}) {
    ADC_CUDA(cudaMalloc((void **)d, nva * sizeof(double)));
    ADC_CUDA(cudaMemset(*d, 0, nva * sizeof(double)));
  }
  ADC_CUDA(cudaMalloc((void **)&c->pipe, 3 * nva * sizeof(double)));
  ADC_CUDA(cudaMemset(c->pipe, 0, 3 * nva * sizeof(double)));
  if (c->nfluxibp) {
    if (!a->pipeht || !a->pipecoef || !a->pipediam) {
      set_error("the mesh has barrier pipes (IBTYPE 5/25) but no PIPEHT/PIPECOEF/PIPEDIAM");
      return ADC_ERR_MESH;
    }
    ADC_CUDA(cudaMemcpy(c->pipe, a->pipeht, nv * sizeof(double), cudaMemcpyHostToDevice));
    ADC_CUDA(cudaMemcpy(c->pipe + nva, a->pipecoef, nv * sizeof(double), cudaMemcpyHostToDevice));
    ADC_CUDA(cudaMemcpy(c->pipe + 2 * nva, a->pipediam, nv * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (c->nfluxib) {
    ADC_CUDA(cudaMemcpy(c->binht, a->barinht, nv * sizeof(double), cudaMemcpyHostToDevice));
    ADC_CUDA(cudaMemcpy(c->bincfsb, a->barincfsb, nv * sizeof(double), cudaMemcpyHostToDevice));
    ADC_CUDA(cudaMemcpy(c->bincfsp, a->barincfsp, nv * sizeof(double), cudaMemcpyHostToDevice));
  }
  const size_t npa = (size_t)c->np;
  ADC_CUDA(cudaMalloc((void **)&c->nib, npa * sizeof(int)));
  ADC_CUDA(cudaMemset(c->nib, 0, npa * sizeof(int)));
  ADC_CUDA(cudaMalloc((void **)&c->nibcnt, npa * sizeof(int)));
  ADC_CUDA(cudaMemset(c->nibcnt, 0, npa * sizeof(int)));
  ADC_CUDA(cudaMalloc((void **)&c->barht, nva * sizeof(double)));
  ADC_CUDA(cudaMalloc((void **)&c->barcf, nva * sizeof(double)));
  ADC_CUDA(cudaMemset(c->barht, 0, nva * sizeof(double)));
  ADC_CUDA(cudaMemset(c->barcf, 0, nva * sizeof(double)));
  if (c->nfluxb) {
    ADC_CUDA(cudaMemcpy(c->barht, a->barlanht, nv * sizeof(double), cudaMemcpyHostToDevice));
    ADC_CUDA(cudaMemcpy(c->barcf, a->barlancfsp, nv * sizeof(double), cudaMemcpyHostToDevice));
  }
  // EtaDisc at the river-radiation nodes from the bound (cold-start) ETA2,
  // cstart.F:1186-1191; ElevDisc is set by the steps
  std::vector<double> ed(nva, 0.0);
  for (int I = 0; I < nv; ++I)
    if (a->lbcodei[I] == 52) ed[I] = a->eta2[bnv[I]];
  ADC_CUDA(cudaMalloc((void **)&c->etadisc_b, nva * sizeof(double)));
  ADC_CUDA(cudaMemcpy(c->etadisc_b, ed.data(), nva * sizeof(double), cudaMemcpyHostToDevice));
  ADC_CUDA(cudaMalloc((void **)&c->elevdisc, nva * sizeof(double)));
  ADC_CUDA(cudaMemset(c->elevdisc, 0, nva * sizeof(double)));
  // zero-normal-gradient entries in ME2GW order (momentum.F:1157-1174)
  std::vector<int> zn, ze;
  std::vector<double> zf;
  for (int J = 0; J < a->nvelme; ++J) {
    const int I = a->me2gw[J] - 1;
    if (I < 0 || I >= nv || a->lbcodei[I] != 40) continue;
    if (!a->nelezng || a->nelezng[I] < 1 || a->nelezng[I] > c->ne) {
      set_error("NEleZNG of boundary entry %d is missing or out of range", I + 1);
      return ADC_ERR_MESH;
    }
    zn.push_back(bnv[I]);
    ze.push_back(a->nelezng[I] - 1);
    zf.push_back(a->zngif1[I]);
    zf.push_back(a->zngif2[I]);
    zf.push_back(a->zngif3[I]);
  }
  c->n_zng = (int)zn.size();
  if ((rc = up_i(&c->zng_node, zn))) return rc;
  if ((rc = up_i(&c->zng_ele, ze))) return rc;
  ADC_CUDA(cudaMalloc((void **)&c->zng_f, std::max<size_t>(zf.size(), 1) * sizeof(double)));
  if (!zf.empty())
    ADC_CUDA(cudaMemcpy(c->zng_f, zf.data(), zf.size() * sizeof(double), cudaMemcpyHostToDevice));
  return ADC_OK;
}

}  // namespace adc

using namespace adc;

extern "C" int adc_set_flux(adc_ctx *c, const adc_flux_t *f) {
  if (!c || !f || f->nffr < 1 || !f->famig || !f->fper || !f->fff || !f->fface || !f->qnam ||
      !f->qnph) {
    set_error("adc_set_flux: at least one flux constituent and every table are required");
    return ADC_ERR_ARG;
  }
  if (!c->nfluxf) {
    set_error("adc_set_flux: the mesh has no specified-flux boundary (IBTYPE 2, 12, 22, 32 or 52)");
    return ADC_ERR_ARG;
  }
  const int nf = f->nffr, nv = c->nvel;
  std::vector<double> cst(4 * (size_t)nf);
  std::memcpy(cst.data(), f->famig, nf * sizeof(double));
  std::memcpy(cst.data() + nf, f->fper, nf * sizeof(double));
  std::memcpy(cst.data() + 2 * nf, f->fff, nf * sizeof(double));
  std::memcpy(cst.data() + 3 * nf, f->fface, nf * sizeof(double));
  if (c->fconst) cudaFree(c->fconst);
  if (c->fqn) cudaFree(c->fqn);
  c->fconst = nullptr;
  c->fqn = nullptr;
  ADC_CUDA(cudaMalloc((void **)&c->fconst, cst.size() * sizeof(double)));
  ADC_CUDA(cudaMemcpy(c->fconst, cst.data(), cst.size() * sizeof(double), cudaMemcpyHostToDevice));
  const size_t nfv = (size_t)nf * nv;
  const int fen = (f->enam && f->enph) ? 1 : 0;
  ADC_CUDA(cudaMalloc((void **)&c->fqn, (fen ? 4 : 2) * nfv * sizeof(double)));
  ADC_CUDA(cudaMemcpy(c->fqn, f->qnam, nfv * sizeof(double), cudaMemcpyHostToDevice));
  ADC_CUDA(cudaMemcpy(c->fqn + nfv, f->qnph, nfv * sizeof(double), cudaMemcpyHostToDevice));
  if (fen) {
    ADC_CUDA(cudaMemcpy(c->fqn + 2 * nfv, f->enam, nfv * sizeof(double), cudaMemcpyHostToDevice));
    ADC_CUDA(cudaMemcpy(c->fqn + 3 * nfv, f->enph, nfv * sizeof(double), cudaMemcpyHostToDevice));
  }
  c->fen = fen;
  c->nffr = nf;
  c->flux_settling_it = f->flux_settling_it;
  c->flux_on = 1;
  c->fser_on = 0;
  drop_graphs(c);   // replayed steps must see the forcing
  return ADC_OK;
}

// Checks a series and uploads its records (width values per record; a
// second table of the same shape when values2 is given, zeros otherwise).
static int series_upload(adc_ctx *c, const adc_series_t *s, int width, const char *what,
                         double **v1, double **v2) {
  if (!s || s->nrec < 2 || !s->values || !(s->interval > 0.0) || !std::isfinite(s->start_time)) {
    set_error("%s: at least two records, a positive interval and a finite start time are required",
              what);
    return ADC_ERR_ARG;
  }
  if (!c->sstate) {
    ADC_CUDA(cudaMalloc((void **)&c->sstate, 2 * sizeof(SeriesState)));
    ADC_CUDA(cudaMemset(c->sstate, 0, 2 * sizeof(SeriesState)));
  }
  const size_t n = (size_t)s->nrec * width;
  for (double **p : {v1, v2})
    if (p && *p) {
      cudaFree(*p);
      *p = nullptr;
    }
  ADC_CUDA(cudaMalloc((void **)v1, n * sizeof(double)));
  ADC_CUDA(cudaMemcpy(*v1, s->values, n * sizeof(double), cudaMemcpyHostToDevice));
  if (v2) {
    ADC_CUDA(cudaMalloc((void **)v2, n * sizeof(double)));
    if (s->values2)
      ADC_CUDA(cudaMemcpy(*v2, s->values2, n * sizeof(double), cudaMemcpyHostToDevice));
    else
      ADC_CUDA(cudaMemset(*v2, 0, n * sizeof(double)));
  }
  return ADC_OK;
}

// cstart.F:207-216 / 227-256: the first two records, ETIME1 = STATIM*86400.
static int series_start(adc_ctx *c, int which, const adc_series_t *s) {
  SeriesState st;
  std::memset(&st, 0, sizeof(st));
  st.t1 = s->start_time;
  st.t2 = st.t1 + s->interval;
  ADC_CUDA(cudaMemcpy(c->sstate + which, &st, sizeof(st), cudaMemcpyHostToDevice));
  drop_graphs(c);
  return ADC_OK;
}

extern "C" int adc_set_elev_series(adc_ctx *c, const adc_series_t *s) {
  if (!c) return ADC_ERR_ARG;
  if (c->neta < 1) {
    set_error("adc_set_elev_series: the mesh has no elevation boundary nodes");
    return ADC_ERR_ARG;
  }
  int rc = series_upload(c, s, c->neta, "adc_set_elev_series", &c->eser, nullptr);
  if (rc) return rc;
  c->eser_nrec = s->nrec;
  c->eser_interval = s->interval;
  c->eser_on = 1;
  return series_start(c, 0, s);
}

extern "C" int adc_set_flux_series(adc_ctx *c, const adc_series_t *s) {
  if (!c) return ADC_ERR_ARG;
  if (!c->nfluxf) {
    set_error("adc_set_flux_series: the mesh has no specified-flux boundary (IBTYPE 2, 12, 22, 32 or 52)");
    return ADC_ERR_ARG;
  }
  int rc = series_upload(c, s, c->nvel, "adc_set_flux_series", &c->fser_q, &c->fser_e);
  if (rc) return rc;
  c->fser_nrec = s->nrec;
  c->fser_interval = s->interval;
  c->flux_settling_it = s->flux_settling_it;
  c->fser_on = 1;
  c->flux_on = 0;
  return series_start(c, 1, s);
}
