// adc_internal.cuh -- device-side data layout shared by the libadcgpu kernels.
//
// HBM layout (one B200, state resident between calls):
//   node arrays      double[NP]  (eta1, eta2, ..., SoA, 0-based node index)
//   element arrays   nm[3*NE] (element-major, 0-based), fdx/fdy[3*NE], areas[NE]
//   node->element    CSR n2e_ptr[NP+1], n2e[3*NE] = 3*e+k sorted by e, so
//                    every per-node sum runs in the reference's element order
//   GWCE matrix      diag[NP] + off-diagonals in sliced ELL (32-row slices,
//                    column-major inside a slice, slot order = NeiTab order)
//   scratch          element contribution buffers, JCG vectors, partials
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cstdio>

#include "../../include/adcgpu.h"

namespace adc {

constexpr int kSlice = 32;            // rows per SELL slice (one warp)
constexpr int kGatherChunk = 8;       // per-node gathers issued together
constexpr int kThreads = 256;
constexpr long long kSpinCycles = 4000000000LL;  // ~2 s at 1.9 GHz

// Device-visible scalar state of the step and of ITPACK.
struct Flags {
  int ncchange;       // NCCHANGE (wetdry.F / gwce.F:430)
  int status;         // ADC_ERR_DIAG on a non-positive diagonal
  int numitr;         // NUMITR of the last solve
  int ier;            // JCG ier of the last solve
  int n_w1_events;    // W1 events of the last wet/dry pass
  int timeout;        // nonzero once a bounded wait expired
  int cursor;         // index of the current step in the step table
  int etadisc_done;   // river radiation: ElevDisc taken (EtaDisc_Fill false, timestep.F:183, 906-926)
  double ep;          // EP (gwce.F:646-650), persists between rebuilds
  double zeta;        // RPARM(1) after the last solve
  double cme;         // RPARM(2) after the last solve
};

// Per-iteration record the JCG scalar block publishes to the row blocks:
// the parcon coefficients, the stop flag and the norm cadence.
struct Rec {
  double c1, c2, c3, c4;
  int halt, need_unorm, in, pad_;
};

// ITPACK common blocks and saved locals (itpackv.F:/itcom1-3/, itjcg save,
// chgcon save) kept between solves.  During a solve the JCG scalar block
// holds them in registers and writes them back at the end.
struct Itp {
  int in, itmax, halt, adapt, q1, chg_ier, isym, pad_;
  double zeta, cme, sme, gamma, rho, gamold, rhoold, delnnm, delsnm, udnm,
      stptst, cmold, srelpr, rparm1;
  Rec rec;
  double dtnrm, unorm;   // peror norms
};

struct Bar {
  unsigned int count;
  unsigned int gen;
};

struct Ctx;
struct Mpnn;

}  // namespace adc

// Host copies of the sliced ELL handed to the solver setup (0-based columns).
struct JcgHostSell {
  const int *sl_ptr, *sl_w, *col, *rlen;
};

// Track state of the parametric vortex (GetHollandStormData's module
// counter and WTRATIO, nws08.F90:68, 114) and this step's storm scalars.
struct VortexState {
  int counter;   // 0-based index of the fix after the current time
  int err;       // set when the run passes the last fix
  double wtratio;
  double x, y, cpress, dpdef, spd, b, rmw, tvx, tvy;
  int calm;      // a CALM fix brackets the time: no wind, background pressure
  int pad_;
};

// Position in a non-periodic boundary series (fort.19 / fort.20): the two
// record times the reference holds (ETIME1/ETIME2, QTIME1/QTIME2), the index
// of the earlier record and this step's interpolation ratio.
struct SeriesState {
  double t1, t2, ratio;
  int k;
  int err;       // set when the run passes the last record
};

// Choice and statistics of the extrapolated JCG initial guess.
struct WarmState {
  int use;         // this step starts from the extrapolated guess
  int pad_;
  long long n_used, n_fallback;
};

struct adc_ctx {
  // sizes
  int np, ne, mnei, neta, nbfr, nvel, nvelme, prec;
  int nslices, nnz_pad, n_obc, n_obc_rhs_nodes, n_me, itmax;
  adc_params_t p;
  int dt_pow2;           // DT is a power of two (its reciprocal is exact)
  double inv_dt;
  adc_arrays_t host;     // bound host arrays (for sync)
  cudaStream_t stream;
  // node data
  double *x, *y, *dp, *tau0, *evm, *fric, *corif;
  int *nneigh;
  // element data
  int *nm;
  double *fdx, *fdy, *areas;
  int *n2e_ptr, *n2e;
  // matrix structure (SELL)
  int *sl_ptr, *sl_w, *col, *rlen;
  int *lhs_src;          // 2 per padded slot: index 6*e+q of the element off-diagonal value, or -1
  int *ell_of_sell;      // host-side sync helper: SELL slot -> (i + np*j) ELL index (device copy unused)
  int *h_ell_of_sell;
  // boundaries
  int *nbd, *is_nbd;     // is_nbd[i] = I index (0-based) or -1
  double *amig, *per, *face, *ff, *emo, *efa;
  int *obc_slot, *obc_zero;   // per (I,J): SELL slot of Coef(nb,IJ) (-1 none), nb-is-NBD flag
  int *obc_rhs_ptr, *obc_rhs_node, *obc_rhs_ent;  // per affected nb: entries I + neta*J, and b
  int *obc_rhs_b;
  int *me_of_node;       // momentum BC entry per node or -1
  int *me_i;             // per momentum BC entry: its boundary entry (NVEL index)
  int *me41_ptr;         // per momentum BC entry: its IBTYPE 41 triples [ptr, ptr+1)
  int *me41_tri;         // (NM2, NM3, NeiTabEle element) triples, 0-based, element -1 = none
  // specified normal flux (flux.cu)
  int nfluxf, flux_on, nffr, n_fx;
  int nfluxrbc;          // radiation (IBTYPE 30) entries present
  int nfluxgbc;          // zero-normal-gradient (IBTYPE 40) entries present
  int nfluxb;            // external barrier (IBTYPE 3/13/23) entries present
  double *barht, *barcf; // BARLANHT, BARLANCFSP per boundary entry
  int nfluxib;           // internal barrier (IBTYPE 4/24/5/25) entries present
  int nfluxibp;          // barriers with cross-barrier pipes (IBTYPE 5/25) present
  double *pipe;          // PIPEHT, PIPECOEF, PIPEDIAM per entry (3 x NVEL)
  int *ibconn;           // per boundary entry: the node across the barrier (0-based)
  int *ibkind;           // per entry: 0 first, 1 last, 2 inner node of its face; -1 none
  double *binht, *bincfsb, *bincfsp;   // BARINHT, BARINCFSB, BARINCFSP per entry
  int *nib;              // NIBNODECODE (NP): receives barrier overflow this step
  int *nibcnt;           // NIBCNT (NP), wetdry.F:813-816
  int n_zng;             // IBTYPE 40 momentum entries, in ME2GW order:
  int *zng_node, *zng_ele;   //   boundary node, NEleZNG (0-based)
  double *zng_f;             //   ZNGIF1-3 (3 per entry)
  int flux_settling_it;  // FluxSettlingIT (river radiation, IBTYPE 52)
  double *elevdisc;      // ElevDisc per boundary entry (IBTYPE 52)
  double *en;            // EN0, EN1, EN2 (NVEL each): specified elevation of IBTYPE 32
  int fen;               // ENAM/ENPH follow QNAM/QNPH in fqn
  double *etadisc_b;     // EtaDisc at the boundary entries' nodes
  // non-periodic boundary series: fort.19 elevations (NETA per record) and
  // fort.20 fluxes and elevations (NVEL per record); sstate[0] elevation,
  // sstate[1] flux
  int eser_on, fser_on, eser_nrec, fser_nrec;
  double eser_interval, fser_interval;
  double *eser, *fser_q, *fser_e;
  SeriesState *sstate;
  double *qn;            // QN0, QN1, QN2 (NVEL each)
  double *qforce;        // per boundary entry: the GWCE line-integral force
  double *fconst, *fqn;  // FAMIG/FPER/FFF/FFACE, then QNAM and QNPH (NFFR x NVEL)
  int *bnv, *blbc;       // boundary entries: node (0-based), LBCODEI
  double *bbl;           // BNDLEN2O3
  double *bcsii, *bsiii; // CSII, SIII per boundary entry (radiation discharge)
  int *fx_node, *fx_ptr, *fx_ent;   // per boundary node: (segment << 1 | side) in order
  int *me_lbc;
  double *me_csi, *me_sii;
  // state
  double *eta1, *eta2, *etas, *uu1, *vv1, *uu2, *vv2, *qx1, *qy1, *qx2, *qy2, *h1, *h2;
  double *tk, *tkm, *totalarea, *alphal, *wsx1, *wsy1, *wsx2, *wsy2, *pr1, *pr2;
  double *gwce_lv, *mom_x, *mom_y;
  int *nodecode, *nnodecode, *noff, *noffold, *mju, *ncele;
  double *diag, *offd, *obccoef;
  // incremental GWCE LHS rebuild: cached element entries and the inputs they
  // were built with, rows to gather again, boundary rows (always gathered)
  // and each row's gathered diagonal
  double *lhs_ebuf, *lhs_al, *diag_gathered;
  int *lhs_nc;
  unsigned char *lhs_dirty, *bc_row;
  // scratch
  double *ebuf;          // element contributions, 9*NE doubles
  double *ebuf2;         // 3*NE doubles (momentum y)
  double *red;           // reduction partials
  // W1 events
  int *ev_cnt;           // per element-block event counts, then their offsets
  int *evu_i;            // unordered W1 events (a, b, element) while they fit a chunk
  double *evu_c;
  int *ev_a, *ev_b;      // per element: NM123, partner (compacted per block)
  double *ev_c;
  int ev_blocks;
  // JCG
  double *ju1, *jw, *soff;
  double4 *jp[2];        // JCG (dtwd, d, d_prev, -) per node, double-buffered
  double *jpart;         // partial dots per block (4 each)
  double *jtri;          // tri(itmax,4)
  adc::Itp *itp;
  adc::Bar *bar;
  void *jlines;          // JCG barrier lines: 2 x 128 B per row block
  int jcg_grid, jcg_rows_blocks;
  // JCG resident variant (block-local indices, halo lists, export flags)
  int jcg_res, jcg_rows_max, jcg_halo_max, jcg_stage_bytes, jcg_stage_wcap;
  size_t jcg_smem;
  unsigned short *jlcol;
  float *soff32;               // FP32 scaled matrix (mixed mode, resident variant)
  double *etas_prev;           // last step's reference guess (ADC_WARM_START)
  WarmState *warm;
  adc::Mpnn *mp;               // learned initial guess (mpnn.cu), built on first use
  int *h_neitab, *h_nneigh;    // host copies of NeiTab/NNeigh (the predictor's 1-ring)
  int *jhalo_ptr, *jhalo_ids;
  unsigned char *jexp;
  // flags / steps
  adc::Flags *flags;
  adc_step_t *steps;     // device step table
  int steps_cap;
  int *numitr_log;
  int numitr_cap;
  // met forcing staging
  double *met_wsx, *met_wsy, *met_pr;
  int met_pending;
  // parametric vortex forcing (NWS = 8)
  int vortex_on;
  adc_vortex_t vpar;
  adc_vortex_fix_t *vfix;
  VortexState *vstate;
  // timing
  cudaEvent_t ev[6];
  cudaEvent_t kev[2 * 6];   // start/end of the kernel spans of adc_kernel_times
  int kmark;                // record kev while capturing the timed single-step graph
  int64_t launches;
  // graph
  cudaGraphExec_t graph;
  int graph_ok;
  cudaGraphExec_t graph1;   // one timed step (adc_timestep), phase events inside
  int graph1_ok, graph1_launches;
  int graph_launches;    // kernel launches per replayed step
  int graph_gen;         // bumped whenever the step's captured form changes
  int jcg_nrb_req;       // requested JCG row blocks (0: the default choice)
  cudaEvent_t run_ev[2];
  double last_run_ms;
};

namespace adc {

// Error bookkeeping (thread-local message).
void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

#define ADC_CUDA(call)                                         \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return adc::cuda_fail(e_, #call);   \
  } while (0)

inline int nblk(long long n, int t = kThreads) { return (int)((n + t - 1) / t); }

// Phase launchers (each returns ADC_OK or an error, records launches).
int launch_shift_friction(adc_ctx *c);
int launch_gwce_lhs(adc_ctx *c);
int launch_gwce_rhs(adc_ctx *c);
int launch_jcg(adc_ctx *c, int eta_update);
int launch_wetdry(adc_ctx *c);
int launch_momentum(adc_ctx *c);

// Drops the captured step graphs (after a change they would not see).
inline void drop_graphs(adc_ctx *c) {
  if (c->graph_ok) cudaGraphExecDestroy(c->graph);
  if (c->graph1_ok) cudaGraphExecDestroy(c->graph1);
  c->graph_ok = 0;
  c->graph1_ok = 0;
  c->graph_gen++;   // graphs that captured this context's step are stale too
}

// Programmatic dependent launch.  Step kernels are launched so that the
// next kernel's grid is set up while the previous one drains; each kernel
// first waits (griddepcontrol.wait) until its predecessor has completed
// and its memory is visible, so nothing runs early.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t stream,
                     Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Kernel spans timed in the single-step graph (adc_kernel_times).
enum KSpan { KS_LHS_ELEM = 0, KS_LHS_GATHER, KS_RHS_ELEM, KS_RHS_GATHER, KS_MOM_ELEM, KS_MOM_NODE };
inline void kmark(adc_ctx *c, int span, int end) {
  if (c->kmark) cudaEventRecordWithFlags(c->kev[2 * span + end], c->stream, cudaEventRecordExternal);
}

// Which parts run in FP32 (ADC_PREC_MIXED selects all of them).
inline bool f32_assembly(const adc_ctx *c) { return c->prec & (ADC_PREC_MIXED | ADC_F32_ASSEMBLY); }
inline bool f32_spmv(const adc_ctx *c) { return c->prec & (ADC_PREC_MIXED | ADC_F32_SPMV); }
inline bool f32_momentum(const adc_ctx *c) { return c->prec & (ADC_PREC_MIXED | ADC_F32_MOMENTUM); }
inline bool any_f32(const adc_ctx *c) { return f32_assembly(c) || f32_spmv(c) || f32_momentum(c); }

// Correctly rounded division by a constant known in advance, after
// Brisebarre, Muller and Raina, "Accelerating correctly rounded
// floating-point division when the divisor is known in advance" (IEEE
// Trans. Computers 53(8), 2004): with zh = RN(1/y), q = RN(x*zh) is
// corrected once by the exact remainder r = x - q*y (one FMA) as
// RN(q + r*zh).  For y = 3*2^k the exact quotient's significand has a
// fractional part of 0, 1/3 or 2/3 ulp, never within 1/6 ulp of a rounding
// midpoint, while the corrected value is within a tiny fraction of an ulp
// of it, so the result is RN(x/y) for finite x in the normal range; an
// exact quotient keeps q itself, so the sign of a zero is kept, and a
// non-finite q (x = +-inf or NaN) is returned as it is, as x/y would give.  The
// library's self-check (adc_selftest_div_const) compares it bit for bit
// with IEEE division on 2^30 random and adversarial inputs per divisor.
// It replaces full divisions in the FP64 element kernels' averages.
__device__ __forceinline__ double div_known(double x, double y, double zh) {
  const double q = x * zh;
  const double r = fma(-q, y, x);
  return (r == 0.0 || !isfinite(q)) ? q : fma(r, zh, q);
}
__device__ __forceinline__ double div3(double x) { return div_known(x, 3.0, 1.0 / 3.0); }
__device__ __forceinline__ double div6(double x) { return div_known(x, 6.0, 1.0 / 6.0); }
__device__ __forceinline__ double div12(double x) { return div_known(x, 12.0, 1.0 / 12.0); }
__device__ __forceinline__ float div3(float x) { return x / 3.0f; }
__device__ __forceinline__ float div6(float x) { return x / 6.0f; }
__device__ __forceinline__ float div12(float x) { return x / 12.0f; }

// Stores K consecutive values per lane (lane l owns out[K*l .. K*l+K-1]
// of the warp's span) as K coalesced 32-wide stores through shared memory
// `sh` (32*K values per warp).  Every lane of the warp must call it;
// `nvalid` lanes carry data.
template <int K, class T>
__device__ __forceinline__ void warp_store_k(T *out, const T (&v)[K], int nvalid, T *sh) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < K; ++k) sh[lane * K + k] = v[k];
  __syncwarp();
#pragma unroll
  for (int m = 0; m < K; ++m) {
    const int idx = m * 32 + lane;
    if (idx < nvalid * K) out[idx] = sh[idx];
  }
  __syncwarp();
}

// Deterministic block reduction of one double (fixed tree).
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace adc
