// step.cu -- libadcgpu host side: bind/upload, the TIMESTEP 2DDI sequence,
// graph replay, host synchronisation and the ITPACK jcg drop-in.
#include "adc_internal.cuh"

#include <cstdio>

#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

namespace adc {

thread_local std::string g_err;

void set_error(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}

int cuda_fail(cudaError_t e, const char *what) {
  set_error("%s: %s", what, cudaGetErrorString(e));
  return ADC_ERR_CUDA;
}

int jcg_setup_grid(adc_ctx *c, const JcgHostSell *h);

// kernels defined in the other translation units
__global__ void k_shift_friction(adc_ctx c, const adc_step_t *steps, const Flags *flags);
__global__ void k_apply_met(adc_ctx c);
__global__ void k_lhs_begin(Flags *f, int *words);
__global__ void k_lhs_drift(adc_ctx c, const int *apply);
__global__ void k_lhs_drift_flush(int *words);
template <class R> __global__ void k_lhs_elem(adc_ctx c, const int *rebuild);
template <class R> __global__ void k_lhs_gather(adc_ctx c, const int *rebuild);
__global__ void k_lhs_ep(adc_ctx c, const int *rebuild, int nparts);
__global__ void k_lhs_bc(adc_ctx c, const int *rebuild);
template <class R> __global__ void k_rhs_elem(adc_ctx c);
template <class R> __global__ void k_rhs_gather(adc_ctx c);
__global__ void k_eta_bc(adc_ctx c, const adc_step_t *steps, const Flags *flags);
__global__ void k_obc_rhs(adc_ctx c);

__global__ void k_step_end(Flags *f, int *numitr_log, int cap) {
  griddep_wait();
  int k = f->cursor;
  if (k < cap) numitr_log[k] = f->numitr;
  f->cursor = k + 1;
}

// Device scratch for the rebuild flag lives after the flags struct.
static int *rebuild_flag(adc_ctx *c) { return (int *)(c->flags + 1); }

int launch_met_vortex(adc_ctx *c);
int launch_flux_forcing(adc_ctx *c);
int launch_flux_rhs(adc_ctx *c);
int flux_tables(adc_ctx *c, const adc_arrays_t *a);
int launch_warm_start(adc_ctx *c);
int launch_predictor_train(adc_ctx *c);

int launch_shift_friction(adc_ctx *c) {
  launch_k(k_shift_friction, nblk(c->np), kThreads, c->stream, *c, c->steps, c->flags);
  c->launches++;
  int rc = launch_met_vortex(c);
  if (rc) return rc;
  if (c->met_pending) {
    launch_k(k_apply_met, nblk(c->np), kThreads, c->stream, *c);
    c->launches++;
  }
  return launch_flux_forcing(c);   // timestep.F:606-613 and 861-880, after the met forcing
}

int launch_gwce_lhs(adc_ctx *c) {
  int *rb = rebuild_flag(c);
  launch_k(k_lhs_begin, 1, 1, c->stream, c->flags, rb);
  int nb = nblk(c->np);
  launch_k(k_lhs_drift, nb, kThreads, c->stream, *c, rb + 2);
  kmark(c, KS_LHS_ELEM, 0);
  if (f32_assembly(c)) {   // FP32 element assembly
    launch_k(k_lhs_elem<float>, nblk(c->ne), kThreads, c->stream, *c, rb);
    kmark(c, KS_LHS_ELEM, 1);
    kmark(c, KS_LHS_GATHER, 0);
    launch_k(k_lhs_gather<float>, nb, kThreads, c->stream, *c, rb);
  } else {
    launch_k(k_lhs_elem<double>, nblk(c->ne), kThreads, c->stream, *c, rb);
    kmark(c, KS_LHS_ELEM, 1);
    kmark(c, KS_LHS_GATHER, 0);
    launch_k(k_lhs_gather<double>, nb, kThreads, c->stream, *c, rb);
  }
  kmark(c, KS_LHS_GATHER, 1);
  launch_k(k_lhs_ep, 1, 1024, c->stream, *c, rb, nb);
  launch_k(k_lhs_bc, nblk((long long)c->np + c->n_obc), kThreads, c->stream, *c, rb);
  c->launches += 6;
  return ADC_OK;
}

int launch_gwce_rhs(adc_ctx *c) {
  kmark(c, KS_RHS_ELEM, 0);
  if (f32_assembly(c)) {
    launch_k(k_rhs_elem<float>, nblk(c->ne), kThreads, c->stream, *c);
    kmark(c, KS_RHS_ELEM, 1);
    kmark(c, KS_RHS_GATHER, 0);
    launch_k(k_rhs_gather<float>, nblk(c->np), kThreads, c->stream, *c);
  } else {
    launch_k(k_rhs_elem<double>, nblk(c->ne), kThreads, c->stream, *c);
    kmark(c, KS_RHS_ELEM, 1);
    kmark(c, KS_RHS_GATHER, 0);
    launch_k(k_rhs_gather<double>, nblk(c->np), kThreads, c->stream, *c);
  }
  kmark(c, KS_RHS_GATHER, 1);
  c->launches += 2;
  int rc = launch_flux_rhs(c);   // gwce.F:1737-1834, before the elevation rows
  if (rc) return rc;
  if (c->neta > 0) {
    launch_k(k_eta_bc, nblk(c->neta), kThreads, c->stream, *c, c->steps, c->flags);
    c->launches++;
    if (c->n_obc_rhs_nodes > 0) {
      launch_k(k_obc_rhs, nblk(c->n_obc_rhs_nodes), kThreads, c->stream, *c);
      c->launches++;
    }
  }
  return ADC_OK;
}

// The whole 2DDI step (TIMESTEP order), without host synchronisation.
static int enqueue_step(adc_ctx *c, bool timed) {
  int rc;
  c->kmark = timed ? 1 : 0;
  if (timed) cudaEventRecordWithFlags(c->ev[0], c->stream, cudaEventRecordExternal);
  if ((rc = launch_shift_friction(c))) return rc;
  if (timed) cudaEventRecordWithFlags(c->ev[1], c->stream, cudaEventRecordExternal);
  if ((rc = launch_gwce_lhs(c))) return rc;
  if ((rc = launch_gwce_rhs(c))) return rc;
  if ((rc = launch_warm_start(c))) return rc;
  if (timed) cudaEventRecordWithFlags(c->ev[2], c->stream, cudaEventRecordExternal);
  if ((rc = launch_jcg(c, 1))) return rc;
  if ((rc = launch_predictor_train(c))) return rc;   // nothing unless training is on
  if (timed) cudaEventRecordWithFlags(c->ev[3], c->stream, cudaEventRecordExternal);
  if ((rc = launch_wetdry(c))) return rc;
  if (timed) cudaEventRecordWithFlags(c->ev[4], c->stream, cudaEventRecordExternal);
  if ((rc = launch_momentum(c))) return rc;
  if (timed) cudaEventRecordWithFlags(c->ev[5], c->stream, cudaEventRecordExternal);
  c->kmark = 0;
  return ADC_OK;
}

template <class T>
static int dalloc(T **p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess) {
    set_error("cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    return ADC_ERR_NOMEM;
  }
  return ADC_OK;
}

template <class T>
static int up(T *d, const T *h, size_t n) {
  if (n == 0) return ADC_OK;
  ADC_CUDA(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice));
  return ADC_OK;
}

template <class T>
static int down(T *h, const T *d, size_t n) {
  if (n == 0 || h == nullptr) return ADC_OK;
  ADC_CUDA(cudaMemcpy(h, d, n * sizeof(T), cudaMemcpyDeviceToHost));
  return ADC_OK;
}

#define TRY(x)                 \
  do {                         \
    int rc_ = (x);             \
    if (rc_) return rc_;       \
  } while (0)

// ---------------------------------------------------------------- bind
struct HostTables {
  std::vector<int> nm, n2e_ptr, n2e, sl_ptr, sl_w, col, rlen, lhs_src, ell_of_sell;
  std::vector<int> is_nbd, nbd, obc_slot, obc_zero, obc_rhs_ptr, obc_rhs_node, obc_rhs_ent,
      obc_rhs_b, me_of_node, me_lbc, me_i;
  std::vector<double> me_csi, me_sii;
  std::vector<int> me41_ptr, me41_tri;   // Galerkin zero-gradient (IBTYPE 41) neighbour triples
  std::vector<int> sell_of_ell;   // ELL (i + np*j), j >= 1 -> SELL idx or -1
};

static int build_tables(const adc_arrays_t *a, HostTables &T, int &nslices, int &nnz_pad) {
  const int np = a->np, ne = a->ne, mnei = a->mnei, neta = a->neta;
  T.nm.resize(3 * (size_t)ne);
  for (int e = 0; e < ne; ++e)
    for (int k = 0; k < 3; ++k) {
      int v = a->nm[e + (size_t)ne * k];
      if (v < 1 || v > np) { set_error("NM(%d,%d) = %d out of range", e + 1, k + 1, v); return ADC_ERR_MESH; }
      T.nm[3 * (size_t)e + k] = v - 1;
    }
  T.n2e_ptr.assign(np + 1, 0);
  for (int e = 0; e < ne; ++e)
    for (int k = 0; k < 3; ++k) T.n2e_ptr[T.nm[3 * (size_t)e + k] + 1]++;
  for (int i = 0; i < np; ++i) T.n2e_ptr[i + 1] += T.n2e_ptr[i];
  T.n2e.resize(3 * (size_t)ne);
  {
    std::vector<int> fill(T.n2e_ptr.begin(), T.n2e_ptr.end() - 1);
    for (int e = 0; e < ne; ++e)
      for (int k = 0; k < 3; ++k) T.n2e[fill[T.nm[3 * (size_t)e + k]]++] = 3 * e + k;
  }
  // sliced ELL of the off-diagonal NeiTab slots
  nslices = (np + kSlice - 1) / kSlice;
  T.rlen.assign(np, 0);
  T.sl_w.assign(nslices, 0);
  T.sl_ptr.assign(nslices + 1, 0);
  for (int i = 0; i < np; ++i) {
    int nn = a->nneigh[i];
    if (nn < 1 || nn > mnei) { set_error("NNeigh(%d) = %d", i + 1, nn); return ADC_ERR_MESH; }
    T.rlen[i] = nn - 1;
    if (a->neitab[i] != i + 1) { set_error("NeiTab(%d,1) is not the node itself", i + 1); return ADC_ERR_MESH; }
    T.sl_w[i / kSlice] = std::max(T.sl_w[i / kSlice], nn - 1);
  }
  for (int s = 0; s < nslices; ++s) T.sl_ptr[s + 1] = T.sl_ptr[s] + T.sl_w[s] * kSlice;
  nnz_pad = T.sl_ptr[nslices];
  T.col.assign(std::max(nnz_pad, 1), 0);
  T.ell_of_sell.assign(std::max(nnz_pad, 1), -1);
  T.sell_of_ell.assign((size_t)np * mnei, -1);
  for (int i = 0; i < np; ++i) {
    int s = i / kSlice, lane = i % kSlice;
    for (int k = 0; k < T.sl_w[s]; ++k) {
      int idx = T.sl_ptr[s] + k * kSlice + lane;
      if (k < T.rlen[i]) {
        int j = a->neitab[i + (size_t)np * (k + 1)];
        if (j < 1 || j > np) { set_error("NeiTab(%d,%d) = %d", i + 1, k + 2, j); return ADC_ERR_MESH; }
        T.col[idx] = j - 1;
        T.ell_of_sell[idx] = i + np * (k + 1);
        T.sell_of_ell[i + (size_t)np * (k + 1)] = idx;
      } else {
        T.col[idx] = i;
      }
    }
  }
  // padded rows of the last slice point at row 0 (never used)
  // LHS contribution map: element off-diagonal value q in 3..8 -> slot
  T.lhs_src.assign(2 * (size_t)std::max(nnz_pad, 1), -1);
  static const int qk[6] = {0, 0, 1, 1, 2, 2}, ql[6] = {0, 1, 0, 1, 0, 1};
  for (int e = 0; e < ne; ++e) {
    for (int t = 0; t < 6; ++t) {
      int k = qk[t], l = ql[t];
      int row = T.nm[3 * (size_t)e + k];
      int J = a->csr_position[e + (size_t)ne * (k + 3 * l)];
      if (J < 2 || J > a->nneigh[row]) { set_error("CSR_POSITION(%d,%d,%d) = %d", e + 1, k + 1, l + 1, J); return ADC_ERR_MESH; }
      int idx = T.sell_of_ell[row + (size_t)np * (J - 1)];
      if (idx < 0) { set_error("CSR slot missing"); return ADC_ERR_MESH; }
      int v = 9 * e + 3 + t;
      if (T.lhs_src[2 * (size_t)idx] < 0) T.lhs_src[2 * (size_t)idx] = v;
      else if (T.lhs_src[2 * (size_t)idx + 1] < 0) T.lhs_src[2 * (size_t)idx + 1] = v;
      else { set_error("edge shared by more than two elements"); return ADC_ERR_MESH; }
    }
  }
  // elevation boundary tables
  T.is_nbd.assign(np, -1);
  T.nbd.resize(std::max(neta, 1));
  for (int I = 0; I < neta; ++I) {
    int b = a->nbd[I] - 1;
    if (b < 0 || b >= np) { set_error("NBD(%d) out of range", I + 1); return ADC_ERR_MESH; }
    T.nbd[I] = b;
    T.is_nbd[b] = I;
  }
  const int nobc = neta * (mnei - 1);
  T.obc_slot.assign(std::max(nobc, 1), -1);
  T.obc_zero.assign(std::max(nobc, 1), 0);
  std::vector<std::vector<std::pair<int, int>>> rhs_lists(np);   // (entry, b)
  for (int I = 0; I < neta; ++I) {
    int b = T.nbd[I];
    for (int J = 2; J <= a->nneigh[b]; ++J) {
      int q = I + neta * (J - 2);
      int nb = a->neitab[b + (size_t)np * (J - 1)] - 1;
      for (int IJ = 2; IJ <= a->nneigh[nb]; ++IJ)
        if (a->neitab[nb + (size_t)np * (IJ - 1)] - 1 == b) {
          T.obc_slot[q] = T.sell_of_ell[nb + (size_t)np * (IJ - 1)];
          T.obc_zero[q] = (T.is_nbd[nb] >= 0) ? 1 : 0;
        }
      if (T.is_nbd[nb] < 0) rhs_lists[nb].push_back({q, b});
    }
  }
  T.obc_rhs_ptr.assign(1, 0);
  for (int i = 0; i < np; ++i) {
    if (rhs_lists[i].empty()) continue;
    T.obc_rhs_node.push_back(i);
    for (auto &pr : rhs_lists[i]) {
      T.obc_rhs_ent.push_back(pr.first);
      T.obc_rhs_b.push_back(pr.second);
    }
    T.obc_rhs_ptr.push_back((int)T.obc_rhs_ent.size());
  }
  // momentum boundary table
  T.me_of_node.assign(np, -1);
  for (int J = 0; J < a->nvelme; ++J) {
    int I = a->me2gw[J] - 1;
    if (I < 0 || I >= a->nvel) { set_error("ME2GW(%d) out of range", J + 1); return ADC_ERR_MESH; }
    int node = a->nbv[I] - 1;
    if (node < 0 || node >= np) { set_error("NBV out of range"); return ADC_ERR_MESH; }
    if (T.me_of_node[node] >= 0) { set_error("node %d has two momentum BC entries", node + 1); return ADC_ERR_MESH; }
    T.me_of_node[node] = J;
    T.me_lbc.push_back(a->lbcodei[I]);
    T.me_i.push_back(I);
    T.me_csi.push_back(a->csii[I]);
    T.me_sii.push_back(a->siii[I]);
  }
  // IBTYPE 41 (momentum.F:864-933): per momentum entry, the ring's
  // (NM2, NM3, NeiTabEle) triples in the order the reference visits them,
  // the wrap-around pair last; NeiTabEle is used positionally as there
  T.me41_ptr.assign(1, 0);
  for (int J = 0; J < a->nvelme; ++J) {
    const int I = a->me2gw[J] - 1;
    if (a->lbcodei[I] == 41) {
      if (!a->neitabele) { set_error("IBTYPE 41 needs NeiTabEle"); return ADC_ERR_MESH; }
      const int node = a->nbv[I] - 1, nn = a->nneigh[node];
      auto NT = [&](int k) { return a->neitab[node + (size_t)np * (k - 1)] - 1; };
      auto TE = [&](int k) { return a->neitabele[node + (size_t)np * (k - 1)] - 1; };
      int nm2 = NT(2);
      const int first = nm2;
      for (int q = 3; q <= nn; ++q) {
        const int nm3 = nm2;
        nm2 = NT(q);
        T.me41_tri.insert(T.me41_tri.end(), {nm2, nm3, TE(q - 2)});
      }
      T.me41_tri.insert(T.me41_tri.end(), {first, nm2, TE(nn - 1)});
    }
    T.me41_ptr.push_back((int)(T.me41_tri.size() / 3));
  }
  return ADC_OK;
}

static int upload_state(adc_ctx *c) {
  const adc_arrays_t *a = &c->host;
  const int np = c->np, ne = c->ne;
  TRY(up(c->eta1, a->eta1, np));
  TRY(up(c->eta2, a->eta2, np));
  TRY(up(c->etas, a->etas, np));
  TRY(up(c->uu1, a->uu1, np));
  TRY(up(c->vv1, a->vv1, np));
  TRY(up(c->uu2, a->uu2, np));
  TRY(up(c->vv2, a->vv2, np));
  TRY(up(c->qx1, a->qx1, np));
  TRY(up(c->qy1, a->qy1, np));
  TRY(up(c->qx2, a->qx2, np));
  TRY(up(c->qy2, a->qy2, np));
  TRY(up(c->h1, a->h1, np));
  TRY(up(c->h2, a->h2, np));
  TRY(up(c->tk, a->tk, np));
  TRY(up(c->tkm, a->tkm, 3 * (size_t)np));
  TRY(up(c->totalarea, a->totalarea, np));
  TRY(up(c->alphal, a->alphal, ne));
  TRY(up(c->wsx1, a->wsx1, np));
  TRY(up(c->wsy1, a->wsy1, np));
  TRY(up(c->wsx2, a->wsx2, np));
  TRY(up(c->wsy2, a->wsy2, np));
  TRY(up(c->pr1, a->pr1, np));
  TRY(up(c->pr2, a->pr2, np));
  TRY(up(c->gwce_lv, a->gwce_lv, np));
  TRY(up(c->mom_x, a->mom_lv_x, np));
  TRY(up(c->mom_y, a->mom_lv_y, np));
  TRY(up(c->nodecode, a->nodecode, np));
  TRY(up(c->nnodecode, a->nnodecode, np));
  TRY(up(c->noff, a->noff, ne));
  TRY(up(c->mju, a->mju, np));
  // COEF(NP,MNEI): column 1 -> diag, other NeiTab slots -> SELL
  std::vector<double> d(np), o(std::max(c->nnz_pad, 1), 0.0);
  for (int i = 0; i < np; ++i) d[i] = a->coef[i];
  for (int idx = 0; idx < c->nnz_pad; ++idx)
    if (c->h_ell_of_sell[idx] >= 0) o[idx] = a->coef[c->h_ell_of_sell[idx]];
  TRY(up(c->diag, d.data(), np));
  TRY(up(c->offd, o.data(), c->nnz_pad));
  {
    // the host COEF is authoritative: no drift pending, and the next rebuild
    // recomputes every element and gathers every row
    int words[4] = {0, 0, 0, 1};
    TRY(up(rebuild_flag(c), words, 4));
    ADC_CUDA(cudaMemset(c->lhs_nc, 0xff, (size_t)c->ne * sizeof(int)));
  }
  TRY(up(c->obccoef, a->obccoef, (size_t)c->neta * (c->mnei - 1)));
  return ADC_OK;
}

static int download_state(adc_ctx *c) {
  adc_arrays_t *a = &c->host;
  const int np = c->np, ne = c->ne;
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  TRY(down(a->eta1, c->eta1, np));
  TRY(down(a->eta2, c->eta2, np));
  TRY(down(a->etas, c->etas, np));
  TRY(down(a->uu1, c->uu1, np));
  TRY(down(a->vv1, c->vv1, np));
  TRY(down(a->uu2, c->uu2, np));
  TRY(down(a->vv2, c->vv2, np));
  TRY(down(a->qx1, c->qx1, np));
  TRY(down(a->qy1, c->qy1, np));
  TRY(down(a->qx2, c->qx2, np));
  TRY(down(a->qy2, c->qy2, np));
  TRY(down(a->h1, c->h1, np));
  TRY(down(a->h2, c->h2, np));
  TRY(down(a->tk, c->tk, np));
  TRY(down(a->tkm, c->tkm, 3 * (size_t)np));
  TRY(down(a->totalarea, c->totalarea, np));
  TRY(down(a->alphal, c->alphal, ne));
  TRY(down(a->wsx1, c->wsx1, np));
  TRY(down(a->wsy1, c->wsy1, np));
  TRY(down(a->wsx2, c->wsx2, np));
  TRY(down(a->wsy2, c->wsy2, np));
  TRY(down(a->pr1, c->pr1, np));
  TRY(down(a->pr2, c->pr2, np));
  TRY(down(a->gwce_lv, c->gwce_lv, np));
  TRY(down(a->mom_lv_x, c->mom_x, np));
  TRY(down(a->mom_lv_y, c->mom_y, np));
  TRY(down(a->nodecode, c->nodecode, np));
  TRY(down(a->nnodecode, c->nnodecode, np));
  TRY(down(a->noff, c->noff, ne));
  TRY(down(a->mju, c->mju, np));
  if (a->coef) {
    // COEF as the reference holds it: apply a drift the last solve left pending
    int *w = rebuild_flag(c);
    launch_k(k_lhs_drift_flush, 1, 1, c->stream, w);
    launch_k(k_lhs_drift, nblk(np), kThreads, c->stream, *c, w + 2);
    ADC_CUDA(cudaGetLastError());
    ADC_CUDA(cudaStreamSynchronize(c->stream));
    std::vector<double> d(np), o(std::max(c->nnz_pad, 1));
    TRY(down(d.data(), c->diag, np));
    TRY(down(o.data(), c->offd, c->nnz_pad));
    std::fill(a->coef, a->coef + (size_t)np * c->mnei, 0.0);
    for (int i = 0; i < np; ++i) a->coef[i] = d[i];
    for (int idx = 0; idx < c->nnz_pad; ++idx)
      if (c->h_ell_of_sell[idx] >= 0) a->coef[c->h_ell_of_sell[idx]] = o[idx];
  }
  TRY(down(a->obccoef, c->obccoef, (size_t)c->neta * (c->mnei - 1)));
  return ADC_OK;
}

void mp_free(adc_ctx *c);

static void free_ctx(adc_ctx *c) {
  if (!c) return;
  mp_free(c);
  delete[] c->h_nneigh;
  delete[] c->h_neitab;
  c->h_nneigh = c->h_neitab = nullptr;
  void **ptrs[] = {
      (void **)&c->x, (void **)&c->y, (void **)&c->dp, (void **)&c->tau0, (void **)&c->evm,
      (void **)&c->fric, (void **)&c->corif, (void **)&c->nneigh, (void **)&c->nm,
      (void **)&c->fdx, (void **)&c->fdy, (void **)&c->areas, (void **)&c->n2e_ptr,
      (void **)&c->n2e, (void **)&c->sl_ptr, (void **)&c->sl_w, (void **)&c->col,
      (void **)&c->rlen, (void **)&c->lhs_src, (void **)&c->nbd, (void **)&c->is_nbd,
      (void **)&c->amig, (void **)&c->per, (void **)&c->face, (void **)&c->ff,
      (void **)&c->emo, (void **)&c->efa, (void **)&c->obc_slot, (void **)&c->obc_zero,
      (void **)&c->obc_rhs_ptr, (void **)&c->obc_rhs_node, (void **)&c->obc_rhs_ent,
      (void **)&c->obc_rhs_b, (void **)&c->me_of_node, (void **)&c->me_lbc,
      (void **)&c->me_csi, (void **)&c->me_sii, (void **)&c->me_i, (void **)&c->me41_ptr,
      (void **)&c->me41_tri, (void **)&c->qn,
      (void **)&c->qforce, (void **)&c->fconst, (void **)&c->fqn, (void **)&c->bnv, (void **)&c->blbc,
      (void **)&c->bbl, (void **)&c->bcsii, (void **)&c->bsiii, (void **)&c->barht, (void **)&c->barcf, (void **)&c->ibconn,
      (void **)&c->ibkind, (void **)&c->binht, (void **)&c->bincfsb, (void **)&c->bincfsp,
      (void **)&c->nib, (void **)&c->nibcnt, (void **)&c->pipe, (void **)&c->elevdisc, (void **)&c->etadisc_b, (void **)&c->en, (void **)&c->zng_node, (void **)&c->zng_ele, (void **)&c->zng_f, (void **)&c->fx_node, (void **)&c->fx_ptr, (void **)&c->fx_ent, (void **)&c->eta1, (void **)&c->eta2,
      (void **)&c->etas, (void **)&c->uu1, (void **)&c->vv1, (void **)&c->uu2, (void **)&c->vv2,
      (void **)&c->qx1, (void **)&c->qy1, (void **)&c->qx2, (void **)&c->qy2, (void **)&c->h1,
      (void **)&c->h2, (void **)&c->tk, (void **)&c->tkm, (void **)&c->totalarea,
      (void **)&c->alphal, (void **)&c->wsx1, (void **)&c->wsy1, (void **)&c->wsx2,
      (void **)&c->wsy2, (void **)&c->pr1, (void **)&c->pr2, (void **)&c->gwce_lv,
      (void **)&c->mom_x, (void **)&c->mom_y, (void **)&c->nodecode, (void **)&c->nnodecode,
      (void **)&c->noff, (void **)&c->noffold, (void **)&c->mju, (void **)&c->ncele,
      (void **)&c->diag, (void **)&c->offd, (void **)&c->obccoef, (void **)&c->lhs_ebuf,
      (void **)&c->lhs_al, (void **)&c->diag_gathered, (void **)&c->lhs_nc, (void **)&c->lhs_dirty,
      (void **)&c->bc_row, (void **)&c->ebuf,
      (void **)&c->ebuf2, (void **)&c->red, (void **)&c->ev_cnt, (void **)&c->ev_a,
      (void **)&c->ev_b, (void **)&c->ev_c, (void **)&c->evu_i, (void **)&c->evu_c, (void **)&c->ju1, (void **)&c->jp[0],
      (void **)&c->jp[1], (void **)&c->jw, (void **)&c->jexp, (void **)&c->jlcol,
      (void **)&c->jhalo_ptr, (void **)&c->jhalo_ids, (void **)&c->soff32, (void **)&c->etas_prev, (void **)&c->warm, (void **)&c->soff, (void **)&c->jpart, (void **)&c->jtri,
      (void **)&c->itp, (void **)&c->bar, (void **)&c->jlines, (void **)&c->flags, (void **)&c->steps,
      (void **)&c->numitr_log, (void **)&c->met_wsx, (void **)&c->met_wsy,
      (void **)&c->met_pr, (void **)&c->vfix, (void **)&c->vstate, (void **)&c->eser,
      (void **)&c->fser_q, (void **)&c->fser_e, (void **)&c->sstate};
  for (void **p : ptrs)
    if (*p) { cudaFree(*p); *p = nullptr; }
  drop_graphs(c);
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto &e : c->run_ev)
    if (e) cudaEventDestroy(e);
  for (auto &e : c->kev)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete[] c->h_ell_of_sell;
  delete c;
}

static int bind_impl(const adc_params_t *p, const adc_arrays_t *a, int prec, adc_ctx **out) {
  if (!p || !a || !out) { set_error("null argument"); return ADC_ERR_ARG; }
  if (a->np <= 0 || a->ne <= 0 || a->mnei < 2 || a->neta < 0 || a->nbfr < 0) {
    set_error("invalid sizes"); return ADC_ERR_ARG;
  }
  if (prec & ~(ADC_PREC_MIXED | ADC_WARM_START | ADC_F32_ASSEMBLY | ADC_F32_SPMV | ADC_F32_MOMENTUM |
               ADC_LEARNED_START)) {
    set_error("bad precision mode %d", prec);
    return ADC_ERR_ARG;
  }
  if (p->itmax < 0 || p->dt <= 0.0) { set_error("invalid parameters"); return ADC_ERR_ARG; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("no CUDA device available");
    return ADC_ERR_CUDA;
  }
  HostTables T;
  int nslices = 0, nnz_pad = 0;
  TRY(build_tables(a, T, nslices, nnz_pad));
  adc_ctx *c = new adc_ctx();
  memset((void *)c, 0, sizeof(*c));
  *out = nullptr;
  c->np = a->np; c->ne = a->ne; c->mnei = a->mnei; c->neta = a->neta; c->nbfr = a->nbfr;
  c->nvel = a->nvel; c->nvelme = a->nvelme; c->prec = prec; c->itmax = p->itmax;
  {
    int ex = 0;
    c->dt_pow2 = (p->dt > 0.0 && std::frexp(p->dt, &ex) == 0.5) ? 1 : 0;
    c->inv_dt = 1.0 / p->dt;
  }
  c->p = *p;
  c->host = *a;
  c->nslices = nslices;
  c->nnz_pad = nnz_pad;
  c->n_obc = a->neta * (a->mnei - 1);
  c->n_obc_rhs_nodes = (int)T.obc_rhs_node.size();
  c->n_me = (int)T.me_lbc.size();
  c->h_ell_of_sell = new int[std::max(nnz_pad, 1)];
  std::copy(T.ell_of_sell.begin(), T.ell_of_sell.end(), c->h_ell_of_sell);
  auto fail = [&](int rc) { free_ctx(c); return rc; };
#define B(x) do { int rc_ = (x); if (rc_) return fail(rc_); } while (0)
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(ADC_ERR_CUDA);
  for (auto &e : c->ev) cudaEventCreate(&e);
  for (auto &e : c->kev) cudaEventCreate(&e);
  for (auto &e : c->run_ev) cudaEventCreate(&e);
  const int np = c->np, ne = c->ne;
  B(dalloc(&c->x, np)); B(up(c->x, a->x, np));
  B(dalloc(&c->y, np)); B(up(c->y, a->y, np));
  B(dalloc(&c->dp, np)); B(up(c->dp, a->dp, np));
  B(dalloc(&c->tau0, np)); B(up(c->tau0, a->tau0var, np));
  B(dalloc(&c->evm, np)); B(up(c->evm, a->evm, np));
  B(dalloc(&c->fric, np)); B(up(c->fric, a->fric, np));
  B(dalloc(&c->corif, np)); B(up(c->corif, a->corif, np));
  B(dalloc(&c->nneigh, np)); B(up(c->nneigh, a->nneigh, np));
  B(dalloc(&c->nm, 3 * (size_t)ne)); B(up(c->nm, T.nm.data(), T.nm.size()));
  B(dalloc(&c->fdx, 3 * (size_t)ne)); B(up(c->fdx, a->fdxe, 3 * (size_t)ne));
  B(dalloc(&c->fdy, 3 * (size_t)ne)); B(up(c->fdy, a->fdye, 3 * (size_t)ne));
  B(dalloc(&c->areas, ne)); B(up(c->areas, a->areas, ne));
  B(dalloc(&c->n2e_ptr, np + 1)); B(up(c->n2e_ptr, T.n2e_ptr.data(), np + 1));
  B(dalloc(&c->n2e, 3 * (size_t)ne)); B(up(c->n2e, T.n2e.data(), T.n2e.size()));
  B(dalloc(&c->sl_ptr, nslices + 1)); B(up(c->sl_ptr, T.sl_ptr.data(), nslices + 1));
  B(dalloc(&c->sl_w, nslices)); B(up(c->sl_w, T.sl_w.data(), nslices));
  B(dalloc(&c->col, std::max(nnz_pad, 1))); B(up(c->col, T.col.data(), T.col.size()));
  const size_t npad = (size_t)nslices * kSlice;   // row arrays read by whole slices
  {
    std::vector<int> rl(npad, 0);
    std::copy(T.rlen.begin(), T.rlen.end(), rl.begin());
    B(dalloc(&c->rlen, npad)); B(up(c->rlen, rl.data(), npad));
  }
  B(dalloc(&c->lhs_src, T.lhs_src.size())); B(up(c->lhs_src, T.lhs_src.data(), T.lhs_src.size()));
  B(dalloc(&c->nbd, T.nbd.size())); B(up(c->nbd, T.nbd.data(), T.nbd.size()));
  B(dalloc(&c->is_nbd, np)); B(up(c->is_nbd, T.is_nbd.data(), np));
  int nbfr = std::max(a->nbfr, 1), neta = std::max(a->neta, 1);
  B(dalloc(&c->amig, nbfr)); B(dalloc(&c->per, nbfr)); B(dalloc(&c->face, nbfr)); B(dalloc(&c->ff, nbfr));
  B(dalloc(&c->emo, (size_t)nbfr * neta)); B(dalloc(&c->efa, (size_t)nbfr * neta));
  if (a->nbfr > 0) {
    B(up(c->amig, a->amig, a->nbfr)); B(up(c->per, a->per, a->nbfr));
    B(up(c->face, a->face, a->nbfr)); B(up(c->ff, a->ff, a->nbfr));
    B(up(c->emo, a->emo, (size_t)a->nbfr * a->neta)); B(up(c->efa, a->efa, (size_t)a->nbfr * a->neta));
  }
  B(dalloc(&c->obc_slot, T.obc_slot.size())); B(up(c->obc_slot, T.obc_slot.data(), T.obc_slot.size()));
  {
    // rows the boundary pass rewrites (elevation-specified rows and the rows
    // holding OBCCoef entries) are gathered on every rebuild
    std::vector<unsigned char> bc(np, 0);
    for (int b : T.nbd) bc[b] = 1;
    for (size_t q = 0; q < T.obc_slot.size(); ++q) {
      const int slot = T.obc_slot[q];
      if (slot < 0) continue;
      int sl = (int)(std::upper_bound(T.sl_ptr.begin(), T.sl_ptr.end(), slot) - T.sl_ptr.begin()) - 1;
      int row = sl * kSlice + (slot - T.sl_ptr[sl]) % kSlice;
      if (row < np) bc[row] = 1;
    }
    B(dalloc(&c->bc_row, np)); B(up(c->bc_row, bc.data(), np));
  }
  B(dalloc(&c->lhs_ebuf, 9 * (size_t)ne)); B(dalloc(&c->lhs_al, ne)); B(dalloc(&c->lhs_nc, ne));
  ADC_CUDA(cudaMemset(c->lhs_nc, 0xff, (size_t)ne * sizeof(int)));   // no element cached yet
  B(dalloc(&c->lhs_dirty, np)); ADC_CUDA(cudaMemset(c->lhs_dirty, 1, np));
  B(dalloc(&c->diag_gathered, np));
  B(dalloc(&c->obc_zero, T.obc_zero.size())); B(up(c->obc_zero, T.obc_zero.data(), T.obc_zero.size()));
  B(dalloc(&c->obc_rhs_ptr, T.obc_rhs_ptr.size())); B(up(c->obc_rhs_ptr, T.obc_rhs_ptr.data(), T.obc_rhs_ptr.size()));
  B(dalloc(&c->obc_rhs_node, std::max<size_t>(T.obc_rhs_node.size(), 1))); B(up(c->obc_rhs_node, T.obc_rhs_node.data(), T.obc_rhs_node.size()));
  B(dalloc(&c->obc_rhs_ent, std::max<size_t>(T.obc_rhs_ent.size(), 1))); B(up(c->obc_rhs_ent, T.obc_rhs_ent.data(), T.obc_rhs_ent.size()));
  B(dalloc(&c->obc_rhs_b, std::max<size_t>(T.obc_rhs_b.size(), 1))); B(up(c->obc_rhs_b, T.obc_rhs_b.data(), T.obc_rhs_b.size()));
  B(dalloc(&c->me_of_node, np)); B(up(c->me_of_node, T.me_of_node.data(), np));
  B(dalloc(&c->me_i, std::max<size_t>(T.me_i.size(), 1))); B(up(c->me_i, T.me_i.data(), T.me_i.size()));
  B(flux_tables(c, a));
  B(dalloc(&c->me_lbc, std::max<size_t>(T.me_lbc.size(), 1))); B(up(c->me_lbc, T.me_lbc.data(), T.me_lbc.size()));
  B(dalloc(&c->me_csi, std::max<size_t>(T.me_csi.size(), 1))); B(up(c->me_csi, T.me_csi.data(), T.me_csi.size()));
  B(dalloc(&c->me_sii, std::max<size_t>(T.me_sii.size(), 1))); B(up(c->me_sii, T.me_sii.data(), T.me_sii.size()));
  B(dalloc(&c->me41_ptr, T.me41_ptr.size())); B(up(c->me41_ptr, T.me41_ptr.data(), T.me41_ptr.size()));
  B(dalloc(&c->me41_tri, std::max<size_t>(T.me41_tri.size(), 1)));
  if (!T.me41_tri.empty()) B(up(c->me41_tri, T.me41_tri.data(), T.me41_tri.size()));
  double **node_f64[] = {&c->eta1, &c->eta2, &c->etas, &c->uu1, &c->vv1, &c->uu2, &c->vv2, &c->qx1,
                         &c->qy1, &c->qx2, &c->qy2, &c->h1, &c->h2, &c->tk, &c->totalarea,
                         &c->wsx1, &c->wsy1, &c->wsx2, &c->wsy2, &c->pr1, &c->pr2, &c->gwce_lv,
                         &c->mom_x, &c->mom_y, &c->diag, &c->ju1, &c->jw, &c->met_wsx,
                         &c->met_wsy, &c->met_pr};
  for (double **q : node_f64) B(dalloc(q, npad));
  B(dalloc(&c->jp[0], npad)); B(dalloc(&c->jp[1], npad));
  ADC_CUDA(cudaMemset(c->etas, 0, npad * sizeof(double)));
  ADC_CUDA(cudaMemset(c->ju1, 0, npad * sizeof(double)));
  ADC_CUDA(cudaMemset(c->jp[0], 0, npad * sizeof(double4)));
  ADC_CUDA(cudaMemset(c->jp[1], 0, npad * sizeof(double4)));
  B(dalloc(&c->tkm, 3 * (size_t)np));
  B(dalloc(&c->alphal, ne));
  int **node_i32[] = {&c->nodecode, &c->nnodecode, &c->mju};
  for (int **q : node_i32) B(dalloc(q, np));
  B(dalloc(&c->noff, ne)); B(dalloc(&c->noffold, ne)); B(dalloc(&c->ncele, ne));
  B(dalloc(&c->offd, std::max(nnz_pad, 1))); B(dalloc(&c->soff, std::max(nnz_pad, 1)));
  if (f32_spmv(c)) B(dalloc(&c->soff32, std::max(nnz_pad, 1)));
  B(dalloc(&c->obccoef, (size_t)std::max(c->n_obc, 1)));
  B(dalloc(&c->ebuf, 9 * (size_t)ne)); B(dalloc(&c->ebuf2, 3 * (size_t)ne));
  B(dalloc(&c->red, 2 * (size_t)nblk(np) + 64));
  if (c->prec & ADC_WARM_START) {
    B(dalloc(&c->etas_prev, npad));
    ADC_CUDA(cudaMemset(c->etas_prev, 0, npad * sizeof(double)));
  }
  if (c->prec & (ADC_WARM_START | ADC_LEARNED_START)) {
    B(dalloc(&c->warm, 1));
    ADC_CUDA(cudaMemset(c->warm, 0, sizeof(WarmState)));
  }
  // host copies of the ring tables, for the learned predictor's graph
  c->h_nneigh = new int[np];
  c->h_neitab = new int[(size_t)np * a->mnei];
  memcpy(c->h_nneigh, a->nneigh, np * sizeof(int));
  memcpy(c->h_neitab, a->neitab, (size_t)np * a->mnei * sizeof(int));
  c->ev_blocks = (ne + 255) / 256;
  B(dalloc(&c->ev_cnt, 2 * ((size_t)c->ev_blocks + 1)));   // counts, then offsets
  B(dalloc(&c->evu_i, 3 * 1024)); B(dalloc(&c->evu_c, 1024));   // one W1 chunk (wetdry.cu)
  B(dalloc(&c->ev_a, (size_t)c->ev_blocks * 256)); B(dalloc(&c->ev_b, (size_t)c->ev_blocks * 256));
  B(dalloc(&c->ev_c, (size_t)c->ev_blocks * 256));
  {
    const JcgHostSell hs{T.sl_ptr.data(), T.sl_w.data(), T.col.data(), T.rlen.data()};
    B(jcg_setup_grid(c, &hs));
  }
  B(dalloc(&c->jpart, 4 * (size_t)c->jcg_grid));
  B(dalloc(&c->jtri, 4 * (size_t)std::max(c->itmax, 2)));
  B(dalloc(&c->itp, 1)); B(dalloc(&c->bar, 1));
  B(dalloc((char **)&c->jlines, 2 * 128 * (size_t)c->jcg_rows_blocks));
  {
    // Flags followed by the rebuild word.
    char *f = nullptr;
    if (cudaMalloc((void **)&f, sizeof(Flags) + 64) != cudaSuccess) return fail(ADC_ERR_NOMEM);
    c->flags = (Flags *)f;
  }
  c->steps_cap = 1;
  B(dalloc(&c->steps, 1));
  c->numitr_cap = 1;
  B(dalloc(&c->numitr_log, 1));
  B(upload_state(c));
  Itp itp;
  memset(&itp, 0, sizeof(itp));
  itp.rparm1 = p->convcr;
  itp.srelpr = DBL_EPSILON;
  itp.itmax = p->itmax;
  B(up(c->itp, &itp, 1));
  Bar bar = {0, 0};
  B(up(c->bar, &bar, 1));
  Flags fl;
  memset(&fl, 0, sizeof(fl));
  fl.ncchange = 1;   // adcirc.F:404: the matrix is built on the first step
  B(up(c->flags, &fl, 1));
  int words[4] = {0, 0, 0, 1};   // rebuild, drift pending/apply, gather every row
  B(up(rebuild_flag(c), words, 4));
  ADC_CUDA(cudaDeviceSynchronize());
#undef B
  *out = c;
  return ADC_OK;
}

static int read_flags(adc_ctx *c, Flags &f) {
  ADC_CUDA(cudaMemcpyAsync(&f, c->flags, sizeof(Flags), cudaMemcpyDeviceToHost, c->stream));
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  if (f.timeout) { set_error("a bounded device-side wait expired"); return ADC_ERR_TIMEOUT; }
  return ADC_OK;
}

static void fill_out(const Flags &f, adc_stepout_t *out) {
  if (!out) return;
  memset(out, 0, sizeof(*out));
  out->numitr = f.numitr;
  out->ier = f.ier;
  out->ncchange = f.ncchange;
  out->status = f.status;
  out->ep = f.ep;
  out->n_w1_events = f.n_w1_events;
  out->zeta = f.zeta;
  out->cme = f.cme;
}

// The step's scalars and a zero cursor, in stream order (the host copies
// are pageable, so both are consumed before the calls return).
static int set_single_step(adc_ctx *c, const adc_step_t *s) {
  if (!s) { set_error("null step"); return ADC_ERR_ARG; }
  ADC_CUDA(cudaMemcpyAsync(c->steps, s, sizeof(adc_step_t), cudaMemcpyHostToDevice, c->stream));
  int zero = 0;
  ADC_CUDA(cudaMemcpyAsync(&c->flags->cursor, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  return ADC_OK;
}

// One timed step.  Without host-supplied met forcing it replays a captured
// graph of the step (phase events included), so the per-step call pays no
// per-kernel launch cost.
static int run_single_step(adc_ctx *c) {
  if (c->met_pending) return enqueue_step(c, true);
  if (!c->graph1_ok) {
    cudaGraph_t g = nullptr;
    int64_t l0 = c->launches;
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    int rc = ADC_OK;
    if (e == cudaSuccess) {
      rc = enqueue_step(c, true);
      cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
      if (e2 != cudaSuccess) e = e2;
    }
    c->graph1_launches = (int)(c->launches - l0);
    c->launches = l0;
    if (e == cudaSuccess && rc == ADC_OK && g) {
      e = cudaGraphInstantiate(&c->graph1, g, 0);
      c->graph1_ok = (e == cudaSuccess);
    }
    if (g) cudaGraphDestroy(g);
    if (!c->graph1_ok)
      fprintf(stderr, "adcgpu: single-step graph not used (%s, rc %d)\n", cudaGetErrorString(e), rc);
    cudaGetLastError();
  }
  if (!c->graph1_ok) return enqueue_step(c, true);
  ADC_CUDA(cudaGraphLaunch(c->graph1, c->stream));
  c->launches += c->graph1_launches;
  return ADC_OK;
}

}  // namespace adc

using namespace adc;

extern "C" {

const char *adc_last_error(void) { return g_err.c_str(); }

int adc_gpu_bind(const adc_params_t *p, const adc_arrays_t *a, int prec, adc_ctx **out) {
  return bind_impl(p, a, prec, out);
}

int adc_gpu_free(adc_ctx *c) {
  if (!c) return ADC_ERR_ARG;
  cudaStreamSynchronize(c->stream);
  free_ctx(c);
  return ADC_OK;
}

int adc_shift_friction(adc_ctx *c, const adc_step_t *s) {
  if (!c) return ADC_ERR_ARG;
  TRY(set_single_step(c, s));
  TRY(launch_shift_friction(c));
  c->met_pending = 0;
  ADC_CUDA(cudaGetLastError());
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  return ADC_OK;
}

int adc_gwce_new(adc_ctx *c, const adc_step_t *s, adc_stepout_t *out) {
  if (!c) return ADC_ERR_ARG;
  TRY(set_single_step(c, s));
  TRY(launch_gwce_lhs(c));
  TRY(launch_gwce_rhs(c));
  TRY(launch_warm_start(c));
  TRY(launch_jcg(c, 1));
  TRY(launch_predictor_train(c));
  ADC_CUDA(cudaGetLastError());
  Flags f;
  TRY(read_flags(c, f));
  fill_out(f, out);
  return f.status;   // ADC_OK, ADC_ERR_DIAG (GWCE) or ADC_ERR_ARG (met track ended)
}

int adc_wetdry(adc_ctx *c, const adc_step_t *s, adc_stepout_t *out) {
  if (!c) return ADC_ERR_ARG;
  TRY(set_single_step(c, s));
  TRY(launch_wetdry(c));
  ADC_CUDA(cudaGetLastError());
  Flags f;
  TRY(read_flags(c, f));
  fill_out(f, out);
  return ADC_OK;
}

int adc_momentum(adc_ctx *c, const adc_step_t *s) {
  if (!c) return ADC_ERR_ARG;
  TRY(set_single_step(c, s));
  TRY(launch_momentum(c));
  ADC_CUDA(cudaGetLastError());
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  return ADC_OK;
}

int adc_timestep(adc_ctx *c, const adc_step_t *s, adc_stepout_t *out) {
  if (!c) return ADC_ERR_ARG;
  TRY(set_single_step(c, s));
  TRY(run_single_step(c));
  c->met_pending = 0;
  ADC_CUDA(cudaGetLastError());
  Flags f;
  TRY(read_flags(c, f));
  fill_out(f, out);
  return f.status;   // ADC_OK, ADC_ERR_DIAG (GWCE) or ADC_ERR_ARG (met track ended)
}

int adc_run(adc_ctx *c, int nsteps, const adc_step_t *steps, int *numitr, adc_stepout_t *last) {
  if (!c || nsteps < 0 || (nsteps > 0 && !steps)) { set_error("bad arguments"); return ADC_ERR_ARG; }
  if (nsteps == 0) return ADC_OK;
  if (c->met_pending) { set_error("adc_run does not take per-step host met forcing"); return ADC_ERR_UNSUPPORTED; }
  if (nsteps > c->steps_cap) {
    cudaFree(c->steps);
    c->steps = nullptr;
    TRY(dalloc(&c->steps, nsteps));
    c->steps_cap = nsteps;
    drop_graphs(c);
  }
  if (nsteps > c->numitr_cap) {
    cudaFree(c->numitr_log);
    c->numitr_log = nullptr;
    TRY(dalloc(&c->numitr_log, nsteps));
    c->numitr_cap = nsteps;
    drop_graphs(c);
  }
  ADC_CUDA(cudaMemcpyAsync(c->steps, steps, nsteps * sizeof(adc_step_t), cudaMemcpyHostToDevice, c->stream));
  int zero = 0;
  ADC_CUDA(cudaMemcpyAsync(&c->flags->cursor, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  if (!c->graph_ok) {
    cudaGraph_t g;
    int64_t l0 = c->launches;
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    int rc = ADC_OK;
    if (e == cudaSuccess) {
      rc = enqueue_step(c, false);
      launch_k(k_step_end, 1, 1, c->stream, c->flags, c->numitr_log, c->numitr_cap);
      e = cudaStreamEndCapture(c->stream, &g);
    }
    c->graph_launches = (int)(c->launches - l0) + 1;
    c->launches = l0;
    if (e == cudaSuccess && rc == ADC_OK) {
      e = cudaGraphInstantiate(&c->graph, g, 0);
      cudaGraphDestroy(g);
      c->graph_ok = (e == cudaSuccess);
    }
    cudaGetLastError();
  }
  ADC_CUDA(cudaEventRecord(c->run_ev[0], c->stream));
  for (int k = 0; k < nsteps; ++k) {
    if (c->graph_ok) {
      ADC_CUDA(cudaGraphLaunch(c->graph, c->stream));
      c->launches += c->graph_launches;
    } else {
      TRY(enqueue_step(c, false));
      launch_k(k_step_end, 1, 1, c->stream, c->flags, c->numitr_log, c->numitr_cap);
      c->launches++;
    }
  }
  ADC_CUDA(cudaEventRecord(c->run_ev[1], c->stream));
  ADC_CUDA(cudaGetLastError());
  Flags f;
  TRY(read_flags(c, f));
  {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->run_ev[0], c->run_ev[1]);
    c->last_run_ms = ms;
  }
  if (numitr) ADC_CUDA(cudaMemcpy(numitr, c->numitr_log, nsteps * sizeof(int), cudaMemcpyDeviceToHost));
  fill_out(f, last);
  return f.status;   // ADC_OK, ADC_ERR_DIAG (GWCE) or ADC_ERR_ARG (met track ended)
}

int adc_sync_to_host(adc_ctx *c) {
  if (!c) return ADC_ERR_ARG;
  return download_state(c);
}

int adc_sync_from_host(adc_ctx *c) {
  if (!c) return ADC_ERR_ARG;
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  return upload_state(c);
}

int adc_set_met(adc_ctx *c, const double *wsx2, const double *wsy2, const double *pr2) {
  if (!c || !wsx2 || !wsy2 || !pr2) return ADC_ERR_ARG;
  if (c->p.nws == 0) { set_error("met forcing given but NWS = 0"); return ADC_ERR_ARG; }
  ADC_CUDA(cudaMemcpyAsync(c->met_wsx, wsx2, c->np * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  ADC_CUDA(cudaMemcpyAsync(c->met_wsy, wsy2, c->np * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  ADC_CUDA(cudaMemcpyAsync(c->met_pr, pr2, c->np * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  c->met_pending = 1;
  return ADC_OK;
}

int adc_phase_times(adc_ctx *c, double *ms_shift, double *ms_gwce, double *ms_jcg,
                    double *ms_wetdry, double *ms_momentum) {
  if (!c) return ADC_ERR_ARG;
  float t[5] = {0, 0, 0, 0, 0};
  for (int k = 0; k < 5; ++k) cudaEventElapsedTime(&t[k], c->ev[k], c->ev[k + 1]);
  if (ms_shift) *ms_shift = t[0];
  if (ms_gwce) *ms_gwce = t[1];
  if (ms_jcg) *ms_jcg = t[2];
  if (ms_wetdry) *ms_wetdry = t[3];
  if (ms_momentum) *ms_momentum = t[4];
  return ADC_OK;
}

int adc_get_scalars(adc_ctx *c, adc_scalars_t *out) {
  if (!c || !out) return ADC_ERR_ARG;
  Flags f;
  TRY(read_flags(c, f));
  Itp it;
  ADC_CUDA(cudaMemcpy(&it, c->itp, sizeof(Itp), cudaMemcpyDeviceToHost));
  memset(out, 0, sizeof(*out));
  out->ncchange = f.ncchange;
  out->q1 = it.q1;
  out->ep = f.ep;
  out->rparm1 = it.rparm1;
  out->rparm2 = it.cme;
  out->vortex_counter = -1;
  out->vortex_wtratio = 0.0;
  if (c->vortex_on) {
    VortexState v;
    ADC_CUDA(cudaMemcpy(&v, c->vstate, sizeof(VortexState), cudaMemcpyDeviceToHost));
    out->vortex_counter = v.counter;
    out->vortex_wtratio = v.wtratio;
  }
  return ADC_OK;
}

int adc_kernel_times(adc_ctx *c, double *ms, int n) {
  if (!c || !ms || n < 0) return ADC_ERR_ARG;
  float t[ADC_NKT] = {0};
  auto span = [&](int k, cudaEvent_t a, cudaEvent_t b) { cudaEventElapsedTime(&t[k], a, b); };
  span(ADC_KT_LHS_ELEM, c->kev[2 * KS_LHS_ELEM], c->kev[2 * KS_LHS_ELEM + 1]);
  span(ADC_KT_LHS_GATHER, c->kev[2 * KS_LHS_GATHER], c->kev[2 * KS_LHS_GATHER + 1]);
  span(ADC_KT_RHS_ELEM, c->kev[2 * KS_RHS_ELEM], c->kev[2 * KS_RHS_ELEM + 1]);
  span(ADC_KT_RHS_GATHER, c->kev[2 * KS_RHS_GATHER], c->kev[2 * KS_RHS_GATHER + 1]);
  span(ADC_KT_JCG, c->ev[2], c->ev[3]);
  span(ADC_KT_WETDRY, c->ev[3], c->ev[4]);
  span(ADC_KT_MOM_ELEM, c->kev[2 * KS_MOM_ELEM], c->kev[2 * KS_MOM_ELEM + 1]);
  span(ADC_KT_MOM_NODE, c->kev[2 * KS_MOM_NODE], c->kev[2 * KS_MOM_NODE + 1]);
  cudaGetLastError();
  for (int k = 0; k < n && k < ADC_NKT; ++k) ms[k] = t[k];
  return ADC_OK;
}

int64_t adc_launch_count(adc_ctx *c) { return c ? c->launches : -1; }

int adc_set_jcg_blocks(adc_ctx *c, int nrb) {
  if (!c || nrb < 0) return ADC_ERR_ARG;
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  drop_graphs(c);
  void **old[] = {(void **)&c->jlcol, (void **)&c->jhalo_ptr, (void **)&c->jhalo_ids,
                  (void **)&c->jexp, (void **)&c->jpart, (void **)&c->jlines};
  for (void **q : old)
    if (*q) { cudaFree(*q); *q = nullptr; }
  const size_t nsl = c->nslices, nnz = c->nnz_pad;
  std::vector<int> sl_ptr(nsl + 1), sl_w(nsl), col(std::max<size_t>(nnz, 1)), rlen(nsl * kSlice);
  ADC_CUDA(cudaMemcpy(sl_ptr.data(), c->sl_ptr, (nsl + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  ADC_CUDA(cudaMemcpy(sl_w.data(), c->sl_w, nsl * sizeof(int), cudaMemcpyDeviceToHost));
  if (nnz) ADC_CUDA(cudaMemcpy(col.data(), c->col, nnz * sizeof(int), cudaMemcpyDeviceToHost));
  ADC_CUDA(cudaMemcpy(rlen.data(), c->rlen, nsl * kSlice * sizeof(int), cudaMemcpyDeviceToHost));
  c->jcg_nrb_req = nrb;
  const JcgHostSell hs{sl_ptr.data(), sl_w.data(), col.data(), rlen.data()};
  TRY(jcg_setup_grid(c, &hs));
  TRY(dalloc(&c->jpart, 4 * (size_t)c->jcg_grid));
  TRY(dalloc((char **)&c->jlines, 2 * 128 * (size_t)c->jcg_rows_blocks));
  return ADC_OK;
}

int adc_jcg_layout(adc_ctx *c, int *row_blocks, int *resident) {
  if (!c) return ADC_ERR_ARG;
  if (row_blocks) *row_blocks = c->jcg_rows_blocks;
  if (resident) *resident = c->jcg_res;
  return ADC_OK;
}

}  // extern "C"

// ------------------------------------------------------------ ensembles
// Independent bound contexts (ensemble members) stepped together: one
// captured graph per time step holds every member's whole step on the
// member's own stream, forked from and joined back into the ensemble's
// stream, so members' kernels overlap on the GPU.
struct adc_ensemble {
  int n;
  adc_ctx **m;
  cudaStream_t root;
  cudaEvent_t fork, t0, t1;
  cudaEvent_t *join;
  cudaGraphExec_t graph;
  int graph_ok;
  long long gen;   // sum of the members' graph generations at capture
  double last_ms;
};

namespace adc {

static long long ens_gen(const adc_ensemble *e) {
  long long g = 0;
  for (int k = 0; k < e->n; ++k) g += e->m[k]->graph_gen;
  return g;
}

static int ens_capture(adc_ensemble *e) {
  cudaGraph_t g = nullptr;
  int rc = ADC_OK;
  cudaError_t err = cudaStreamBeginCapture(e->root, cudaStreamCaptureModeThreadLocal);
  if (err != cudaSuccess) return cuda_fail(err, "ensemble capture");
  cudaEventRecord(e->fork, e->root);
  for (int k = 0; k < e->n && rc == ADC_OK; ++k) {
    adc_ctx *c = e->m[k];
    cudaStreamWaitEvent(c->stream, e->fork, 0);
    int64_t l0 = c->launches;
    rc = enqueue_step(c, false);
    launch_k(k_step_end, 1, 1, c->stream, c->flags, c->numitr_log, c->numitr_cap);
    c->graph_launches = (int)(c->launches - l0) + 1;
    c->launches = l0;
    cudaEventRecord(e->join[k], c->stream);
    cudaStreamWaitEvent(e->root, e->join[k], 0);
  }
  cudaError_t e2 = cudaStreamEndCapture(e->root, &g);
  if (err == cudaSuccess) err = e2;
  if (err == cudaSuccess && rc == ADC_OK) err = cudaGraphInstantiate(&e->graph, g, 0);
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
  if (rc) return rc;
  if (err != cudaSuccess) return cuda_fail(err, "ensemble graph");
  e->graph_ok = 1;
  e->gen = ens_gen(e);
  return ADC_OK;
}

}  // namespace adc

extern "C" {

int adc_ensemble_create(int n, adc_ctx *const *ctxs, adc_ensemble **out) {
  if (n <= 0 || !ctxs || !out) { set_error("adc_ensemble_create: bad arguments"); return ADC_ERR_ARG; }
  for (int k = 0; k < n; ++k)
    if (!ctxs[k] || ctxs[k]->met_pending) { set_error("adc_ensemble_create: member %d not usable", k); return ADC_ERR_ARG; }
  adc_ensemble *e = new adc_ensemble();
  memset((void *)e, 0, sizeof(*e));
  e->n = n;
  e->m = new adc_ctx *[n];
  e->join = new cudaEvent_t[n];
  for (int k = 0; k < n; ++k) e->m[k] = ctxs[k];
  cudaError_t err = cudaStreamCreateWithFlags(&e->root, cudaStreamNonBlocking);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaEventCreate(&e->t0);
  if (err == cudaSuccess) err = cudaEventCreate(&e->t1);
  for (int k = 0; k < n && err == cudaSuccess; ++k) err = cudaEventCreateWithFlags(&e->join[k], cudaEventDisableTiming);
  if (err != cudaSuccess) {
    adc_ensemble_free(e);
    return cuda_fail(err, "adc_ensemble_create");
  }
  *out = e;
  return ADC_OK;
}

int adc_ensemble_free(adc_ensemble *e) {
  if (!e) return ADC_ERR_ARG;
  if (e->root) cudaStreamSynchronize(e->root);
  if (e->graph_ok) cudaGraphExecDestroy(e->graph);
  for (int k = 0; k < e->n; ++k)
    if (e->join && e->join[k]) cudaEventDestroy(e->join[k]);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->t0) cudaEventDestroy(e->t0);
  if (e->t1) cudaEventDestroy(e->t1);
  if (e->root) cudaStreamDestroy(e->root);
  delete[] e->join;
  delete[] e->m;
  delete e;
  return ADC_OK;
}

int adc_ensemble_run(adc_ensemble *e, int nsteps, const adc_step_t *steps, int *numitr,
                     adc_stepout_t *last) {
  if (!e || nsteps < 0 || (nsteps > 0 && !steps)) { set_error("bad arguments"); return ADC_ERR_ARG; }
  if (nsteps == 0) return ADC_OK;
  for (int k = 0; k < e->n; ++k) {
    adc_ctx *c = e->m[k];
    if (nsteps > c->steps_cap) {
      cudaFree(c->steps);
      c->steps = nullptr;
      TRY(dalloc(&c->steps, nsteps));
      c->steps_cap = nsteps;
      drop_graphs(c);
    }
    if (nsteps > c->numitr_cap) {
      cudaFree(c->numitr_log);
      c->numitr_log = nullptr;
      TRY(dalloc(&c->numitr_log, nsteps));
      c->numitr_cap = nsteps;
      drop_graphs(c);
    }
    ADC_CUDA(cudaMemcpyAsync(c->steps, steps, nsteps * sizeof(adc_step_t), cudaMemcpyHostToDevice, c->stream));
    int zero = 0;
    ADC_CUDA(cudaMemcpyAsync(&c->flags->cursor, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    ADC_CUDA(cudaEventRecord(e->join[k], c->stream));
    ADC_CUDA(cudaStreamWaitEvent(e->root, e->join[k], 0));
  }
  if (e->graph_ok && e->gen != ens_gen(e)) {
    cudaGraphExecDestroy(e->graph);
    e->graph_ok = 0;
  }
  if (!e->graph_ok) TRY(ens_capture(e));
  ADC_CUDA(cudaEventRecord(e->t0, e->root));
  for (int s = 0; s < nsteps; ++s) {
    ADC_CUDA(cudaGraphLaunch(e->graph, e->root));
    for (int k = 0; k < e->n; ++k) e->m[k]->launches += e->m[k]->graph_launches;
  }
  ADC_CUDA(cudaEventRecord(e->t1, e->root));
  ADC_CUDA(cudaStreamSynchronize(e->root));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e->t0, e->t1);
  e->last_ms = ms;
  int status = ADC_OK;
  for (int k = 0; k < e->n; ++k) {
    adc_ctx *c = e->m[k];
    Flags f;
    TRY(read_flags(c, f));
    if (numitr) ADC_CUDA(cudaMemcpy(numitr + (size_t)k * nsteps, c->numitr_log, nsteps * sizeof(int), cudaMemcpyDeviceToHost));
    if (last) fill_out(f, last + k);
    if (f.status && !status) status = f.status;
  }
  return status;
}

double adc_ensemble_last_ms(adc_ensemble *e) { return e ? e->last_ms : -1.0; }


double adc_last_run_ms(adc_ctx *c) { return c ? c->last_run_ms : -1.0; }

}  // extern "C"
