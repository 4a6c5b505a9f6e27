/*
 * adcgpu.h -- C ABI of libadcgpu, a B200-native (sm_100a) implementation of
 * ADCIRC's per-time-step 2DDI hot path: GWCE assembly, ITPACK JCG solve,
 * wetting/drying and the lumped explicit momentum update.
 *
 * Conventions are those of the Fortran module arrays the reference hands
 * to these routines: column-major storage, 1-based node and element
 * numbers, INTEGER = int32_t, REAL(8) = double.  Every entry point is
 * extern "C" with plain pointers so a Fortran host binds it through
 * ISO_C_BINDING (include/adcgpu_iface.F90) and Python through ctypes.
 *
 * Entry points that allocate device memory: adc_gpu_bind (device mirrors),
 * adc_set_vortex, adc_set_flux, adc_set_elev_series and adc_set_flux_series
 * (forcing tables), adc_set_predictor and the ensemble calls, adc_jcg
 * (staging for one solve) and the self-check; adc_jcg_noalloc allocates
 * nothing.  Errors are
 * returned as status codes; the library never calls exit().
 */
#ifndef ADCGPU_H
#define ADCGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define ADC_OK 0
#define ADC_ERR_DIAG 1        /* GWCE diagonal <= 0: gwce.F:678-707 terminates */
#define ADC_ERR_ARG (-1)      /* invalid argument or size */
#define ADC_ERR_MESH (-2)     /* inconsistent mesh tables */
#define ADC_ERR_CUDA (-3)     /* CUDA runtime error (message: adc_last_error) */
#define ADC_ERR_NOMEM (-4)    /* device allocation failed */
#define ADC_ERR_TIMEOUT (-5)  /* a bounded device-side wait expired */
#define ADC_ERR_UNSUPPORTED (-6) /* option the library does not implement */

/* precision modes for adc_gpu_bind */
#define ADC_PREC_FP64 0       /* every kernel in FP64, reference arithmetic */
#define ADC_PREC_MIXED 1      /* FP32 assembly/SpMV/momentum, FP64 reductions */
#define ADC_WARM_START 2      /* flag OR'ed into the mode: extrapolated JCG initial
                                 guess with fallback to the reference guess */
/* Single FP32 components (flags OR'ed into the mode; ADC_PREC_MIXED is all
 * three).  CG dot products, norms, the stopping test, the eta update and
 * the state stay FP64 in every mode. */
#define ADC_F32_ASSEMBLY 4    /* GWCE LHS and RHS element terms and their gathers */
#define ADC_F32_SPMV 8        /* the JCG matrix the iterations stream (FP64 products) */
#define ADC_F32_MOMENTUM 16   /* momentum element terms and their gather */
#define ADC_LEARNED_START 32  /* flag OR'ed into the mode: JCG starts from the learned
                                 predictor's guess (adc_set_predictor) when its initial
                                 residual is smaller than the reference guess's */

/* Model parameters (fort.15 values and derived switches). */
typedef struct {
  double dt;             /* DTDP */
  double g;              /* gravity, constants.F90:45 */
  double a00, b00, c00;  /* GWCE time weights, read_input.F:2995 */
  double h0, velmin;     /* wet/dry, read_input.F:3006 */
  double slim;           /* slope limiter, global.F:796 */
  double hbreak, ftheta, fgamma; /* hybrid friction, nodalattr.F:509-511 */
  double convcr;         /* JCG tolerance, RPARM(1) (gwce.F:150) */
  double prbckgrnd_mh2o; /* background pressure in m of water, wind.F:354 */
  int ifnlfa, ifnlct, ifnlcat; /* adcirc.F:287-384 */
  int nolifa;            /* 2 = wetting/drying active (wetdry.F:204) */
  int iflinbf, ifnlbf, ifhybf; /* nodalattr.F:1975-1987 */
  int itmax;             /* JCG ITMAX, IPARM(1) */
  int nws;               /* nonzero: met forcing terms are active */
  int ifwind;            /* adcirc.F:391 */
  int isldia;            /* ITPACK output level IPARM(2) (no output is produced) */
  int pad_;
} adc_params_t;

/* Pointers to the host arrays of module MESH / GLOBAL / BOUNDARIES /
 * NodalAttributes.  adc_gpu_bind copies them to the device; state arrays
 * are written back only by adc_sync_to_host. */
typedef struct {
  int np, ne, mnei, neta, nbfr, nvel, nvelme;
  int nbou;                      /* NBOU; with nvell below, needed only for internal barriers */
  const double *x, *y, *dp;      /* (NP) */
  const int *nm;                 /* NM(NE,3) */
  const int *nneigh;             /* NNeigh(NP) */
  const int *neitab;             /* NeiTab(NP,MNEI), 0 = padding */
  const double *fdxe, *fdye;     /* FDXE(3,NE), FDYE(3,NE) */
  const double *areas;           /* AREAS(NE) = 2 x element area */
  const int *csr_position;       /* CSR_POSITION(NE,3,2) */
  const double *tau0var, *evm, *fric, *corif; /* (NP) */
  const int *nbd;                /* NBD(NETA) elevation-specified nodes */
  const double *amig, *per, *face, *ff;       /* (NBFR) */
  const double *emo, *efa;       /* EMO(NBFR,NETA), EFA(NBFR,NETA) [rad] */
  const int *nbv, *lbcodei;      /* (NVEL) */
  const double *csii, *siii;     /* (NVEL) */
  const int *me2gw;              /* (NVELME) */
  const double *bndlen2o3;       /* (NVEL) 2/3 of each boundary segment's length */
  double *eta1, *eta2, *etas;
  double *uu1, *vv1, *uu2, *vv2, *qx1, *qy1, *qx2, *qy2, *h1, *h2;
  double *tk, *tkm;              /* TK(NP), TKM(3,NP) */
  int *nodecode, *nnodecode, *noff, *mju;
  double *totalarea, *alphal;
  double *wsx1, *wsy1, *wsx2, *wsy2, *pr1, *pr2;
  double *coef;                  /* COEF(NP,MNEI) */
  double *obccoef;               /* OBCCoef(NETA,MNEI-1) */
  double *gwce_lv, *mom_lv_x, *mom_lv_y;
  /* zero-normal-gradient entries (IBTYPE 40, mesh.F:2434-2512): the element
   * holding each entry's fictitious interior node and its interpolation
   * factors (adc_zng_setup); NEleZNG = 0 off IBTYPE 40 entries */
  const int *nelezng;            /* NEleZNG(NVEL), 1-based */
  const double *zngif1, *zngif2, *zngif3;   /* (NVEL) */
  const int *neitabele;          /* NeiTabEle(NP,MNEI), 1-based, 0 = none (IBTYPE 41) */
  /* external barriers (IBTYPE 3/13/23, mesh.F:2570-2574): crest height above
   * datum and the supercritical discharge coefficient per boundary entry;
   * NULL when the mesh has none */
  const double *barlanht, *barlancfsp;   /* (NVEL) */
  /* internal barriers (IBTYPE 4/24 and 5/25, mesh.F:2140-2240, 2577-2594): the node
   * across the barrier (IBCONN, 1-based), crest height and the subcritical
   * and supercritical discharge coefficients per boundary entry, front face
   * then back face of each barrier segment; NVELL(NBOU) as mesh.F leaves it
   * (islands closed, barrier segments in pairs).  NULL without internal
   * barriers. */
  const int *ibconn;
  const double *barinht, *barincfsb, *barincfsp;   /* (NVEL) */
  const int *nvell;                                 /* (NBOU) */
  /* cross-barrier pipes of IBTYPE 5/25 barriers (mesh.F:2586-2594): crown
   * height, friction coefficient and diameter per entry; NULL without them */
  const double *pipeht, *pipecoef, *pipediam;      /* (NVEL) */
} adc_arrays_t;

/* Per-step scalars TIMESTEP computes before the hot path (timestep.F:257-353). */
typedef struct {
  int it;
  int pad_;
  double timeloc, timeh, rampelev, rampmete;
  double rampextflux;    /* RampExtFlux, the ramp of specified boundary fluxes */
  double rampintflux;    /* RampIntFlux, the ramp of barrier overflow (IBTYPE 3/13/23) */
} adc_step_t;

/* Periodic specified normal flux on flux boundaries (IBTYPE 2, 12, 22, 32, 52):
 * the fort.15 flux constituents timestep.F:861-880 sums each step. */
typedef struct {
  int nffr;              /* NFFR > 0 constituents */
  int flux_settling_it;  /* FluxSettlingIT = INT(FluxSettlingTime*86400/DTDP),
                            timestep.F:243-245: river-radiation (IBTYPE 52) entries
                            take their discharge elevation at this step and add
                            the radiation term after it (gwce.F:1805-1815) */
  const double *famig;   /* FAMIG(NFFR), rad/s */
  const double *fper;    /* FPER(NFFR), s (0: no whole-period removal) */
  const double *fff;     /* FFF(NFFR), nodal factors */
  const double *fface;   /* FFACE(NFFR), rad */
  const double *qnam;    /* QNAM(NFFR,NVEL), normal flux per unit width, m^2/s */
  const double *qnph;    /* QNPH(NFFR,NVEL), rad */
  const double *enam;    /* ENAM(NFFR,NVEL), m: elevation constituents of coupled
                            flux/radiation entries (IBTYPE 32); NULL when there are none */
  const double *enph;    /* ENPH(NFFR,NVEL), rad */
} adc_flux_t;

/* One fix of a parametric-vortex track: the fields of a fort.22 best-track
 * line that HollandGet consumes (nws08.F90:827-878), in mesh units.  The
 * reference reads longitude/latitude in degrees (ICS=2); this library runs
 * the Cartesian meshes of the path, so the centre is in mesh coordinates
 * (m) and distances are Euclidean. */
typedef struct {
  double time;    /* CastTime: seconds since cold start */
  double x, y;    /* storm centre (Lon, Lat) in mesh coordinates, m */
  double cpress;  /* CPress: central pressure, Pa */
  double vmax;    /* Spd: maximum sustained 10 m wind, m/s */
  double rmw;     /* RMW: radius to maximum winds, km */
  double tvx, tvy;/* TVX, TVY: storm translation velocity, m/s */
} adc_vortex_fix_t;

/* Holland vortex forcing (NWS = 8; HollandGet nws08.F90:562-717 with the
 * radial-velocity-weighted background wind, the limited B of BCalc, no
 * inflow angle, and the NWS = 8 stress of wind.F:1172-1198 with capped
 * Garratt drag wind.F:514-539). */
typedef struct {
  int nfix;               /* number of track fixes (>= 2), times increasing */
  int avg_minute;         /* windspeed_averaging_minute: 1 applies one2ten */
  int hemisphere;         /* sign(1, lat) of the reference: +1 north, -1 south */
  int pad_;
  double start_time;      /* TimeLoc at cold start: picks the first fix pair (NWS08INIT) */
  double bladj;           /* BLAdj, boundary-layer adjustment (fort.15) */
  double rho_air;         /* rhoAir, kg/m^3 (constants.F90 default 1.293) */
  double wind_mult;       /* WindMultiplier (nws08Control) */
  double drag_limit;      /* WindDragLimit (wind.F default 0.0035) */
  const adc_vortex_fix_t *fix;
} adc_vortex_t;

/* fort.22 reader for NWS = 8 (readBestTrackData, nws08.F90:884-1098): the
 * ATCF best-track lines (BEST, OFCL, CALM) as track fixes.  Times are
 * seconds since the wind reference time of the fort.15 NWS = 8 record
 * (TIMECONV, global.F:1556-1583); the centre is projected to mesh
 * coordinates with the CPP projection about (SLAM0, SFEA0) that ICS = 1
 * meshes use (mesh.F:3409-3418); pressure, wind and radius units and the
 * translation velocity (uvtrans, wind/vortex.F:1174-1200) are the
 * reference's.  A CALM line gives a fix with a negative cpress. */
typedef struct {
  int irefyr, irefmo, irefday, irefhr;   /* wind reference time (fort.15) */
  double slam0, sfea0;                   /* CPP projection centre, degrees (fort.15) */
  double rnday;                          /* the track must reach RNDAY days; <= 0: no check */
} adc_fort22_opts_t;

/* With fix == NULL sets *nfix to the number of track times; otherwise fills
 * up to *nfix fixes (ADC_ERR_ARG if the track has more) and sets *nfix.
 * ADC_ERR_ARG on a missing or malformed file, an unknown line type, a
 * forecast line without central pressure or Rmax, or a track that ends
 * before RNDAY (the reference's fatal errors, nws08.F90:1017-1094). */
int adc_fort22_read(const char *path, const adc_fort22_opts_t *opts, int *nfix,
                    adc_vortex_fix_t *fix);

/* Host-visible results of a step or phase. */
typedef struct {
  int numitr;       /* NUMITR = IPARM(1) after JCG (gwce.F:2005) */
  int ier;          /* JCG error flag (itpackv.F: 11, 12, 13, 401, 402) */
  int ncchange;     /* NCCHANGE after wet/dry (wetdry.F:1413-1430) */
  int status;       /* ADC_OK or ADC_ERR_DIAG */
  double ep;        /* EP, RMS of the GWCE diagonal (gwce.F:646-650) */
  double zeta;      /* RPARM(1) after the solve (itpackv.F:394 overwrite) */
  double cme;       /* RPARM(2), eigenvalue estimate */
  int n_w1_events;  /* W1 wetting events that raised TK (wetdry.F:593-618) */
  int pad_;
} adc_stepout_t;

/* ------------------------------------------------------------------ */
/* Drop-in for ITPACK JCG.                                             */
/* ------------------------------------------------------------------ */

/* Replaces `subroutine jcg (n,ndim,maxnz,jcoef,coef,rhs,u,iwksp,nw,wksp,
 * iparm,rparm,ier)`, itpackv.F:63-64, called from gwce.F:2003-2004.
 * Same arguments, by reference.  coef/jcoef/rhs come back unscaled as the
 * reference leaves them (itpackv.F:430); u returns the solution; iparm(1)
 * the iteration count; rparm(1) is overwritten on non-convergence
 * (itpackv.F:394).  Mixed-sign diagonals (ITPACK's isym switch,
 * itpackv.F:2417) return ier = 903 without solving. */
void adc_jcg(const int *n, const int *ndim, const int *maxnz, int *jcoef,
             double *coef, double *rhs, double *u, int *iwksp, const int *nw,
             double *wksp, int *iparm, double *rparm, int *ier);

/* Replaces `subroutine dfault (iparm,rparm)`, itpackv.F:1070. */
void adc_dfault(int *iparm, double *rparm);

/* Clears the ITPACK state that persists between jcg calls (the saved q1
 * flag of itjcg, itpackv.F:459-604) to its program-start value. */
void adc_jcg_reset(void);

/* jcg for callers that may not allocate device memory: a host that owns
 * every device byte through its own pool, or one that runs under a fixed
 * device-memory budget.  No counterpart in the reference: same arguments
 * and results as adc_jcg, but every device buffer is carved from one
 * file-scope __device__ array of 32 MiB that each GPU loading the library
 * holds until exit.  Systems needing more than about
 * n*(20*(maxnz-1)+112) bytes + 32 bytes per ITMAX (checked exactly before
 * any device work) return ier = 905.  The first call on a device resolves
 * the array's address.  Calls share the array: calls whose GPU work
 * overlaps race.  The call is synchronous (cudaMemcpy/cudaMemset on the
 * legacy default stream); it makes no cudaMalloc/cudaFree, no stream
 * creation and no host heap allocation. */
void adc_jcg_noalloc(const int *n, const int *ndim, const int *maxnz, int *jcoef,
                     double *coef, double *rhs, double *u, int *iwksp, const int *nw,
                     double *wksp, int *iparm, double *rparm, int *ier);

/* ------------------------------------------------------------------ */
/* Device-resident 2DDI step (state stays in HBM between calls).       */
/* ------------------------------------------------------------------ */

typedef struct adc_ctx adc_ctx;

/* Binds the module arrays once after ADCIRC_Init (adcirc.F:113-411) and
 * uploads them.  prec is ADC_PREC_FP64 or an OR of ADC_PREC_MIXED,
 * ADC_F32_* and ADC_WARM_START. */
int adc_gpu_bind(const adc_params_t *p, const adc_arrays_t *a, int prec, adc_ctx **out);
int adc_gpu_free(adc_ctx *ctx);

/* TIMESTEP glue before the GWCE: H init at it==1 (timestep.F:231-237),
 * time-level shift and load-vector zeroing (:375-416), bottom friction
 * (nodalattr.F:2399-2413) and the TKM copy (nodalattr.F:2700-2704). */
int adc_shift_friction(adc_ctx *ctx, const adc_step_t *s);

/* Replaces GWCE_New(IT,ITIME_BGN,TimeLoc,TimeH), gwce.F:237, called via
 * solveGWCE (gwce.F:166, timestep.F:1069).  Fills numitr/ier/status/ep. */
int adc_gwce_new(adc_ctx *ctx, const adc_step_t *s, adc_stepout_t *out);

/* Replaces computeWettingAndDrying(it), wetdry.F:140, timestep.F:1088,
 * followed by the H2 update of timestep.F:1097-1099.  Fills ncchange. */
int adc_wetdry(adc_ctx *ctx, const adc_step_t *s, adc_stepout_t *out);

/* Replaces Mom_Eqs_New_NC(), momentum.F:166, via solveMomentumEq
 * (momentum.F:118, timestep.F:1103). */
int adc_momentum(adc_ctx *ctx, const adc_step_t *s);

/* The four calls above in TIMESTEP order for one step. */
int adc_timestep(adc_ctx *ctx, const adc_step_t *s, adc_stepout_t *out);

/* Runs nsteps consecutive steps without host round trips (one captured
 * CUDA graph replayed per step).  numitr[k] (optional, host) receives
 * NUMITR of step k; last receives the outputs of the final step. */
int adc_run(adc_ctx *ctx, int nsteps, const adc_step_t *steps, int *numitr,
            adc_stepout_t *last);

/* Copies device state to the bound host arrays (output/hotstart steps). */
int adc_sync_to_host(adc_ctx *ctx);
/* Re-uploads the bound host state arrays (after a host-side change). */
int adc_sync_from_host(adc_ctx *ctx);

/* Supplies this step's met forcing WSX2/WSY2/PR2 (getMeteorologicalForcing,
 * timestep.F:651) from host arrays of length NP; applied after the shift. */
int adc_set_met(adc_ctx *ctx, const double *wsx2, const double *wsy2, const double *pr2);

/* Replaces getMeteorologicalForcing for NWS = 8 (timestep.F:651,
 * wind.F:1172-1198): uploads a vortex track once; every later step (and
 * adc_run's replayed steps) then forms WSX2/WSY2/PR2 on the device from the
 * track interpolated to TimeLoc (GetHollandStormData, nws08.F90:827-878).
 * Requires NWS != 0 in the bound parameters; nfix < 2 or times that do not
 * increase give ADC_ERR_ARG.  A step past the last fix sets the step status
 * to ADC_ERR_ARG (the reference terminates there). */
int adc_set_vortex(adc_ctx *ctx, const adc_vortex_t *vortex);

/* ------------------------------------------------------------------ */
/* ADCIRC text files at the path's edges (host only; no GPU needed).    */
/* ------------------------------------------------------------------ */

/* fort.14 mesh (read14, mesh.F:319-581).  dims = {NP, NE, NOPE, NETA,
 * NBOU, NVEL}, NVEL counting one line per node (one per pair for internal
 * barriers).  Node labels map to 1..NP in file order, as read14 does.  The
 * barrier records (IBTYPE 3/4/5 families) come from adc_fort14_barriers and
 * adc_fort14_internal_barriers; periodic (94) and VEW (64) segments return
 * ADC_ERR_UNSUPPORTED. */
int adc_fort14_dims(const char *path, int dims[6]);
/* title receives up to 80 characters plus NUL; nm is NM(NE,3); nbdv (NETA)
 * and nbvv (NVEL) are the concatenated segment node lists, segment
 * lengths in nvdll (NOPE) and nvell (NBOU). */
int adc_fort14_read(const char *path, char *title, double *x, double *y, double *dp, int *nm,
                    int *nvdll, int *nbdv, int *nvell, int *ibtype, int *nbvv);
/* Writes the same tables (every double to 17 significant digits). */
int adc_fort14_write(const char *path, const char *title, int np, int ne, const double *x,
                     const double *y, const double *dp, const int *nm, int nope, const int *nvdll,
                     const int *nbdv, int nbou, const int *nvell, const int *ibtype,
                     const int *nbvv);
/* External barrier segments (IBTYPE 3/13/23) carry BARLANHT and BARLANCFSP
 * on each node line (mesh.F:460-473): adc_fort14_barriers returns them per
 * flux-boundary node (NVEL, in file order, 0 elsewhere), and
 * adc_fort14_write_barriers writes a mesh that has such segments. */
int adc_fort14_barriers(const char *path, double *barlanht, double *barlancfsp);
/* Internal barrier segments (IBTYPE 4/24, and 5/25 with pipes) list pairs:
 * the node, the node across the barrier, BARINHT, BARINCFSB, BARINCFSP and
 * for 5/25 PIPEHT, PIPECOEF, PIPEDIAM (mesh.F:479-524); a pair counts twice
 * in the file's NVEL.  adc_fort14_read's nbvv holds the front nodes (nvell
 * counts pairs); adc_fort14_internal_barriers returns IBCONN (1-based) and
 * the values per nbvv entry, 0 elsewhere (the pipe arrays may be NULL). */
int adc_fort14_internal_barriers(const char *path, int *ibconn, double *barinht,
                                 double *barincfsb, double *barincfsp, double *pipeht,
                                 double *pipecoef, double *pipediam);
int adc_fort14_write_barriers(const char *path, const char *title, int np, int ne,
                              const double *x, const double *y, const double *dp, const int *nm,
                              int nope, const int *nvdll, const int *nbdv, int nbou,
                              const int *nvell, const int *ibtype, const int *nbvv,
                              const double *barlanht, const double *barlancfsp,
                              const int *ibconn, const double *barinht,
                              const double *barincfsb, const double *barincfsp,
                              const double *pipeht, const double *pipecoef,
                              const double *pipediam);

/* fort.15 model parameters of a 2DDI run (READ_INPUT, read_input.F:
 * 949-4566), positional records in read_input's order plus the namelist
 * values the path uses (&wetDryControl slim, &metControl WindDragLimit,
 * &nws08Control).
 * Angles read_input converts on reading (FACE, EFA, FFACE, QNPH, ENPH,
 * FACET) are returned in radians.  IM other than 0/10/111111, NWS other
 * than 0/+-8, and station lists in external .151 files return
 * ADC_ERR_UNSUPPORTED; malformed records ADC_ERR_ARG with the record
 * number in adc_last_error(). */
typedef struct {
  int nout, nspool;      /* NOUT*, NSPOOL* */
  double touts, toutf;   /* TOUTS*, TOUTF* (days) */
} adc_output_spec_t;

typedef struct {
  char rundes[88], runid[88];
  int nfover, nabout, nscreen, ihot, ics, im;
  int nolibf, nolifa, nolica, nolicat, nwp, ncor;
  int ntip, nws, nramp, nodedrymin, nodewetmin, storm_number;
  int irefyr, irefmo, irefday, irefhr;             /* NWS = 8 wind record */
  int ntif, nbfr, nffr, nfreq;
  int nstae, nstav, nstac, nstam;
  int nhainc, nhase, nhasv, nhage, nhagv, nhstar;
  int nhsinc, ititer, isldia, itmax;
  int has_slim, has_wind_drag_limit;               /* namelist values found */
  double bladj, g, tau0, tau0_min, tau0_max, dtdp, statim, reftim, rnday;
  double dramp, dramp_extflux, flux_settling_time, dramp_intflux, dramp_elev, dramp_tip,
      dramp_mete, dramp_wrad, dunramp_mete;        /* days */
  double a00, b00, c00, h0, velmin, slam0, sfea0;
  double tau, cf, hbreak, ftheta, fgamma, eslm, eslc, cori, anginn;
  double thas, thaf, fmv, convcr;
  double slim, wind_drag_limit;                    /* defaults 1e9, 0.0035 */
  adc_output_spec_t oute, outv, outc, outm, outge, outgv, outgc, outgw;
  /* &nws08Control (readNws08Namelist, nws08.F90:318-413): the values the
   * Holland path uses; a namelist that selects another vortex model,
   * background wind, B calculation, inflow angle or latitude-dependent
   * angle returns ADC_ERR_UNSUPPORTED */
  int has_nws08, windspeed_averaging_minute;       /* default 1 */
  double wind_multiplier;                          /* default 1 */
} adc_fort15_t;

/* Caller-owned tables adc_fort15_read fills; any pointer may be NULL (a
 * first call with tables = NULL returns the counts NTIF, NBFR, NFFR, NFREQ
 * and the station counts).  Tags are 16 bytes per entry, NUL-terminated. */
typedef struct {
  double *tpk, *amigt, *etrf, *fft, *facet;     /* (NTIF) */
  double *amig, *ff, *face;                     /* (NBFR) */
  double *emo, *efa;                            /* EMO(NBFR,NETA), EFA(NBFR,NETA) */
  double *famig, *fff, *fface;                  /* (NFFR) */
  double *qnam, *qnph, *enam, *enph;            /* QNAM(NFFR,NVEL) ...; 0 off flux nodes */
  double *hafreq, *haff, *haface;               /* (NFREQ); HAFACE in degrees */
  double *xel, *yel, *xev, *yev, *xem, *yem;    /* station coordinates */
  char *tiptag, *bountag, *fbountag, *namefr;
} adc_fort15_tables_t;

/* neta: NETA of the fort.14; lbcodei (NVEL): LBCODEI of every flux-boundary
 * node in the reference's order (adc_boundary_setup's), which decides
 * where the flux records are and how many items each holds. */
int adc_fort15_read(const char *path, int neta, int nvel, const int *lbcodei, adc_fort15_t *out,
                    const adc_fort15_tables_t *tables);
/* Writes the same records in the same order (reals to 17 significant
 * digits, angles in degrees as the file holds them; NWP = 0), so that
 * adc_fort15_read gives back the same values; the namelists only when
 * their has_* flag is set. */
int adc_fort15_write(const char *path, const adc_fort15_t *p, int neta, int nvel,
                     const int *lbcodei, const adc_fort15_tables_t *tables);

/* Full-domain ASCII output files fort.63 (irtype 1) and fort.64 (irtype 2):
 * the header of header63/64 (globalio.F:1005-1085) and one record per call
 * as writeFullFormat/storeOne/storeTwo write them (globalio.F:544-643,
 * 802-930).  With nodecode, dry nodes get `alternate` (-99999 in the
 * reference's elevation output). */
int adc_fort6x_header(const char *path, const char *rundes, const char *runid, const char *agrid,
                      int ndsets, int np, double dt_out, int nspool, int irtype);
int adc_fort6x_append(const char *path, double timeloc, int it, int np, const double *v1,
                      const double *v2, const int *nodecode, double alternate);

/* The reference's own binary hotstart file (fort.67/fort.68, writeHotstart
 * write_output.F:4900-5154, read by hstart.F:500-560) for a serial 2DDI run
 * without harmonic analysis or wave radiation stress: 8-byte direct-access
 * records (header, ETA1, ETA2, EtaDisc, UU2, VV2, CH1 when IM = 10,
 * NODECODE, NOFF, the zero pads and output counters).  adc_fort67_read with
 * np = ne = 0 only fills the header fields; otherwise np and ne must match
 * the file and the arrays are filled (etadisc and ch1 may be NULL).  A host
 * derives H1, H2, ETAS, QX2 and QY2 from them as hstart.F:529-533, 764-768
 * does, then binds or calls adc_sync_from_host. */
typedef struct {
  int im, it, np, ne;
  double timeloc;
  double *eta1, *eta2, *etadisc, *uu2, *vv2, *ch1;   /* (NP) */
  int *nodecode, *noff;                               /* (NP), (NE) */
} adc_fort67_t;
int adc_fort67_write(const char *path, const adc_fort67_t *h);
int adc_fort67_read(const char *path, adc_fort67_t *h);

/* Hotstart: the counterparts of the reference's fort.67/68 dump
 * (write_output.F:4429-5582) and load (hstart.F:47-2048), in this
 * library's own binary format.  The file holds every array and scalar the
 * device step carries between steps (state, the GWCE matrix and EP, ITPACK's
 * persistent scalars, a pending unscal drift, vortex and warm-start state),
 * so a run resumed from it continues bit for bit.  adc_hotstart_read needs
 * a context bound to the same mesh and mode (and, with a vortex, one on
 * which adc_set_vortex was called); it returns ADC_ERR_ARG, with the
 * reason in adc_last_error(), for any other file. */
int adc_hotstart_write(adc_ctx *ctx, const char *path);
int adc_hotstart_read(adc_ctx *ctx, const char *path);

/* Self-check (no reference counterpart): counts, over n generated inputs
 * per divisor, where the library's division by the constants 3, 6 and 12
 * (used in the FP64 element kernels) differs in any bit from IEEE division. */
int adc_selftest_div_const(long long n, unsigned long long seed, long long *mismatches);

/* Specified normal flux (NFLUXF = 1, IBTYPE 2/12/22 with NFFR > 0): uploads
 * the flux constituents once; every later step forms QN2 on the device
 * (timestep.F:861-880) after shifting QN0 <- QN1 <- QN2 (timestep.F:606-613),
 * the GWCE gains the boundary flux integral (gwce.F:1737-1834) and the
 * momentum equation the specified normal velocity -QN2/H2 (momentum.F:
 * 815-856).  Without a call the fluxes stay zero.  ADC_ERR_ARG if the mesh
 * has no flux boundary or nffr < 1.  Radiation boundaries (IBTYPE 30) need
 * no call: every step takes their discharge from the latest velocity
 * (timestep.F:932-940) and the GWCE boundary integral the radiation force
 * (gwce.F:1783-1790).  River-radiation entries (IBTYPE 52) take the flux
 * constituents of this call and, after flux_settling_it, the radiation term
 * against the discharge elevation of that step (gwce.F:1805-1815); the
 * flux-settling ramps themselves are the caller's adc_step_t values
 * (timestep.F:314-345).  Zero-normal-gradient entries (IBTYPE 40) need the
 * NEleZNG/ZNGIF tables of adc_zng_setup in adc_arrays_t.  Coupled
 * flux/radiation entries (IBTYPE 32) take their elevation constituents from
 * enam/enph (gwce.F:1792-1797); Galerkin zero-gradient entries (IBTYPE 41)
 * need NeiTabEle (adc_mesh_neitabele) in adc_arrays_t.  Code 64 is refused
 * at bind with ADC_ERR_UNSUPPORTED. */
int adc_set_flux(adc_ctx *ctx, const adc_flux_t *flux);

/* A non-periodic boundary time series: the records of a fort.19 (elevations)
 * or fort.20 (normal fluxes) after its interval line, one record every
 * `interval` seconds from `start_time`.  The reference reads one record
 * ahead as the run passes each record time and interpolates linearly
 * between the two it holds; here the whole file is in HBM and one device
 * thread per step advances the same pair of record times. */
typedef struct {
  int nrec;               /* records (>= 2) */
  int flux_settling_it;   /* fort.20 series only: FluxSettlingIT (IBTYPE 52) */
  double interval;        /* ETIMINC / FTIMINC, s */
  double start_time;      /* STATIM*86400: ETIME1 / QTIME1 at cold start */
  const double *values;   /* fort.19: ESBIN, NETA per record; fort.20: QNIN,
                             NVEL per record, 0 at entries without a flux record */
  const double *values2;  /* fort.20: ENIN at IBTYPE 32 entries, NVEL per record,
                             NULL when there are none; unused for fort.19 */
} adc_series_t;

/* Non-periodic elevation boundary (NPEBC, a fort.19 beside the fort.15;
 * read_input.F:1893-1898, cstart.F:198-217): every step adds
 * RampElev*(ESBIN1 + ETRATIO*(ESBIN2 - ESBIN1)) to the periodic boundary
 * elevation (gwce.F:1659-1674).  ADC_ERR_ARG without elevation boundary
 * nodes; a run past the last record sets ADC_ERR_ARG in the step status
 * (the reference stops at the end of fort.19). */
int adc_set_elev_series(adc_ctx *ctx, const adc_series_t *series);
/* Non-periodic normal flux (NFFR = 0 or -1, fort.20; cstart.F:227-258): QN2
 * = RampExtFlux*(QNIN1 + QTRATIO*(QNIN2 - QNIN1)) and EN2 likewise at every
 * entry (timestep.F:882-903) in place of the periodic constituents of
 * adc_set_flux.  ADC_ERR_ARG without flux boundaries. */
int adc_set_flux_series(adc_ctx *ctx, const adc_series_t *series);

/* fort.19 / fort.20 readers: the interval line, then records as the
 * reference's list-directed READs take them (one READ per value of ESBIN;
 * per entry of code 2/12/22 one value of QNIN, per entry of code 32 QNIN and
 * ENIN).  With values == NULL only *nrec and *interval are set (the full
 * records in the file); otherwise the first *nrec records are stored,
 * entries of other codes at 0.  Negative on a missing or malformed file. */
int adc_fort19_read(const char *path, int neta, int *nrec, double *interval, double *esbin);
int adc_fort20_read(const char *path, int nvel, const int *lbcodei, int *nrec, double *interval,
                    double *qnin, double *enin);

/* No reference counterpart (the reference always starts JCG from ETAS as
 * GWCE_New leaves it, gwce.F:2002-2004).  With ADC_WARM_START in the bind
 * mode, counts of the steps that started from the extrapolated guess and of
 * those that fell back to the reference guess. */
int adc_warm_start_stats(adc_ctx *ctx, long long *used, long long *fallback);

/* Scalars the device step carries from one step to the next that live in
 * the reference's modules: NCChange (gwce.F:430, wetdry.F:1430), EP
 * (gwce.F:646-650), RPARM(1:2) after the last solve (itpackv.F:394, 442),
 * itjcg's SAVEd q1 flag (itpackv.F:459-604) and NWS = 8's track position
 * bestTrackCounter/WTRATIO (nws08.F90:68, 114, 827-878).  Together with the
 * arrays adc_sync_to_host writes they are the whole step-to-step state, so a
 * host (or a checker) can continue a run from them. */
typedef struct {
  int ncchange;        /* NCChange: nonzero rebuilds the GWCE matrix next step */
  int q1;              /* itjcg's q1 (skip the |u| norm in the stopping test) */
  int vortex_counter;  /* 0-based index of the track fix after the current time */
  int pad_;
  double ep;           /* EP of the last matrix rebuild */
  double rparm1;       /* RPARM(1), zeta (overwritten on non-convergence) */
  double rparm2;       /* RPARM(2), cme: the eigenvalue estimate */
  double vortex_wtratio; /* WTRATIO used for the storm position */
} adc_scalars_t;

int adc_get_scalars(adc_ctx *ctx, adc_scalars_t *out);

/* Learned JCG initial guess (no reference counterpart; the reference starts
 * from ETAS as GWCE_New leaves it, gwce.F:1846-1850, 2002-2004).  A
 * message-passing network over each node's NeiTab ring (input layer 9 -> 64,
 * three layers h' = ReLU(Ws h + Wn mean_ring(h) + b) of width 64, a linear
 * head) predicts a correction s_out * out to that guess at wet nodes off
 * the elevation boundary, from the normalised eta^k, ETAS, u, v, depth, wet
 * flag, p - p_background and wind stress.  BF16 weights and activations,
 * FP32 accumulation on the tensor cores.  Parameters are a flat FP32 array
 * of adc_predictor_nparams() values: W_in[64][16] (inputs 0-8, column 9 the
 * bias, 10-15 zero), per layer Ws[64][64], Wn[64][64], b[64], then
 * w_out[64], b_out, feature means[9], feature scales[9], s_out.
 * adc_set_predictor uploads them (and builds the predictor on first use);
 * with ADC_LEARNED_START in the bind mode every later step starts JCG from
 * the prediction when its initial residual is the smaller one
 * (adc_warm_start_stats counts the choices).  adc_predictor_train(on, lr)
 * trains the network on the device after every step's solve on that
 * step's (features, solved ETAS), Adam on the Huber loss (threshold 3)
 * of the normalised correction; without ADC_LEARNED_START the steps keep the reference guess,
 * so the pairs are the plain solver's.  The predictor is not part of the
 * hotstart file. */
int adc_predictor_nparams(void);
int adc_set_predictor(adc_ctx *ctx, const float *params, int nparams);
int adc_get_predictor(adc_ctx *ctx, float *params, int nparams);
int adc_predictor_train(adc_ctx *ctx, int on, float lr);
/* loss: mean Huber loss of the normalised error of the last training step; adam_steps:
 * updates so far. */
int adc_predictor_stats(adc_ctx *ctx, double *loss, long long *adam_steps);
/* Runs the forward pass on the current device state; guess (NP doubles)
 * receives the predicted ETAS, hidden3 (optional, NP*64 floats) the last
 * hidden layer. */
int adc_predictor_forward(adc_ctx *ctx, double *guess, float *hidden3);
/* The gradient of the last training step, in the parameter layout. */
int adc_predictor_gradient(adc_ctx *ctx, float *grad, int nparams);
/* The gradient of the training loss for the current device state and a
 * given solved ETAS (NP doubles), without updating the weights (a check of
 * the backward pass). */
int adc_predictor_gradient_at(adc_ctx *ctx, const double *target, float *grad, int nparams);

/* Device time of the phases of the last adc_timestep/adc_run (ms). */
int adc_phase_times(adc_ctx *ctx, double *ms_shift, double *ms_gwce, double *ms_jcg,
                    double *ms_wetdry, double *ms_momentum);

/* Device time (ms) of single kernels and passes of the last adc_timestep
 * (events inside its captured step graph), in this order; n entries are
 * written.  No reference counterpart (measurement only). */
#define ADC_KT_LHS_ELEM 0     /* GWCE matrix element terms (gwce.F:427-592) */
#define ADC_KT_LHS_GATHER 1   /* their node-centric gather into COEF */
#define ADC_KT_RHS_ELEM 2     /* GWCE load-vector element terms (gwce.F:1000-1615) */
#define ADC_KT_RHS_GATHER 3   /* their gather into GWCE_LV */
#define ADC_KT_JCG 4          /* the JCG solve (itpackv.F:63-604), all kernels */
#define ADC_KT_WETDRY 5       /* computeWettingAndDrying + H2 (wetdry.F:140-1652) */
#define ADC_KT_MOM_ELEM 6     /* momentum element terms (momentum.F:298-699) */
#define ADC_KT_MOM_NODE 7     /* momentum nodal solve (momentum.F:713-1182) */
#define ADC_NKT 8
int adc_kernel_times(adc_ctx *ctx, double *ms, int n);

/* JCG launch shape of a bound context (no reference counterpart): the
 * persistent solver's row blocks (0 restores the default choice) and
 * whether the resident variant (row vectors in shared memory) is used.
 * adc_set_jcg_blocks rebuilds the solver's tables; results do not depend
 * on it beyond the dot products' summation tree. */
int adc_set_jcg_blocks(adc_ctx *ctx, int row_blocks);
int adc_jcg_layout(adc_ctx *ctx, int *row_blocks, int *resident);

/* Ensembles (no reference counterpart; the reference runs one mesh per
 * process, adcirc.F:475-476): n independent bound contexts stepped
 * together.  Every replayed time step is one captured CUDA graph holding
 * each member's whole step on the member's own stream, so the members'
 * kernels overlap on the GPU.  All members take the same step table (same
 * DT and start time).  numitr (optional) receives NUMITR[member][step],
 * last (optional) each member's outputs after the final step; the return
 * is the first nonzero member status.  A member's later per-context calls
 * (adc_run, adc_timestep, adc_sync_to_host ...) stay valid. */
typedef struct adc_ensemble adc_ensemble;
int adc_ensemble_create(int n, adc_ctx *const *members, adc_ensemble **out);
int adc_ensemble_run(adc_ensemble *ens, int nsteps, const adc_step_t *steps, int *numitr,
                     adc_stepout_t *last);
/* Device time of the last adc_ensemble_run (ms, CUDA events). */
double adc_ensemble_last_ms(adc_ensemble *ens);
int adc_ensemble_free(adc_ensemble *ens);

/* Number of kernel launches issued by the library since bind. */
int64_t adc_launch_count(adc_ctx *ctx);

/* Device time (CUDA events on the library's stream) of the step loop of
 * the last adc_run, excluding its host uploads and readback (ms). */
double adc_last_run_ms(adc_ctx *ctx);

/* Message of the last error (thread-local). */
const char *adc_last_error(void);

/* ------------------------------------------------------------------ */
/* Host-side mesh tables (reference: mesh.F, built once at init).      */
/* ------------------------------------------------------------------ */
int adc_mesh_geometry(int np, int ne, const double *x, const double *y, int *nm,
                      double *fdxe, double *fdye, double *areas);
int adc_mesh_mnei(int np, int ne, const int *nm);
int adc_mesh_neighb(int np, int ne, int mnei, const double *x, const double *y,
                    const int *nm, int *nneigh, int *neitab, int *neimax);
int adc_mesh_csr_positions(int np, int ne, int mnei, const int *nm, const int *neitab,
                           int neimax, int *csr_position);
int adc_boundary_setup(int np, const double *x, const double *y, int nbou,
                       const int *ibtype, const int *seg_ptr, const int *seg_nodes,
                       double cos_inner, int nvel_max, int *nvel, int *nbv,
                       int *lbcodei, double *csii, double *siii, int *nvelme,
                       int *me2gw, double *bndlen2o3);
/* NeiTabEle (NEIGHB, mesh.F:3110-3131, 3248-3283): each node's elements in
 * the order of its NeiTab ring, packed from the front. */
int adc_mesh_neitabele(int np, int ne, int mnei, const int *nm, const int *nneigh,
                       const int *neitab, int *neitabele);
/* Zero-normal-gradient (IBTYPE 40) fictitious nodes (mesh.F:2434-2512):
 * NEleZNG and the interpolation factors ZNGIF1-3 per boundary entry. */
int adc_zng_setup(int np, int ne, const double *x, const double *y, const int *nm, int mnei,
                  const int *nneigh, const int *neitab, const double *areas, int nvel,
                  const int *nbv, const int *lbcodei, const double *csii, const double *siii,
                  int *nelezng, double *zngif1, double *zngif2, double *zngif3);
/* Cold-start wet/dry state (cstart.F:1332-1427) and totalAreaCalc
 * (mesh.F:3360-3400). */
int adc_coldstart(int np, int ne, int nolifa, double h0, const double *dp, const int *nm,
                  const double *areas, double *eta1, double *eta2, int *nnodecode,
                  int *nodecode, int *noff, int *mju, double *totalarea);

#ifdef __cplusplus
}
#endif
#endif
