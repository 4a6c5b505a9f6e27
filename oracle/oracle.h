/*
 * oracle.h -- CPU oracle for the ADCIRC 2DDI time-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a serial FP64 restatement of the
 * reference Fortran (adcirc v56.2.1) used as the checker for the CUDA
 * library.  Only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * --impl reference legs of bench.py may load it.  The product library
 * (adcirc_b200/csrc, include/adcgpu.h) never links or calls it.
 *
 * Parity status: the reference is Fortran and no Fortran compiler exists
 * on the build or GPU hosts, and the reference ships no golden vectors for
 * this path (its acceptance suite lives outside the repository).  The
 * oracle is therefore pinned by mathematical known-answer tests (lake at
 * rest, direct sparse solve, symmetry, mass balance) and by line-by-line
 * citation, not by reference outputs: "parity unpinned" against the
 * reference binary.
 *
 * Layout conventions follow the Fortran module arrays the reference
 * binds: column-major, node/element indices 1-based, INTEGER = int32,
 * REAL(8) = double.  The struct layout is identical to adc_arrays_t /
 * adc_params_t in include/adcgpu.h so one harness can feed both.
 */
#ifndef ADC_ORACLE_H
#define ADC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double dt;            /* DTDP */
  double g;             /* gravity (constants.F90:45, 9.80665) */
  double a00, b00, c00; /* GWCE time weights */
  double h0, velmin;    /* wet/dry thresholds (read_input.F:3006) */
  double slim;          /* slope-limiter parameter (global.F:796) */
  double hbreak, ftheta, fgamma; /* hybrid friction (nodalattr.F:509-511) */
  double convcr;        /* JCG tolerance RPARM(1) */
  double prbckgrnd_mh2o;/* background pressure, m of water (wind.F:354) */
  int ifnlfa, ifnlct, ifnlcat;  /* nonlinear switches (adcirc.F:287-384) */
  int nolifa;           /* 2 = wetting and drying on */
  int iflinbf, ifnlbf, ifhybf;  /* friction law flags (nodalattr.F:1975-1987) */
  int itmax;            /* JCG ITMAX */
  int nws;              /* nonzero when met forcing is applied */
  int ifwind;           /* adcirc.F:391 */
  int isldia;           /* ITPACK output level (IPARM(2)) */
  int pad_;
} orc_params_t;

typedef struct {
  int np, ne, mnei, neta, nbfr, nvel, nvelme, nbou;
  /* mesh.F */
  const double *x, *y, *dp;
  const int *nm;            /* NM(NE,3) */
  const int *nneigh;        /* NNeigh(NP) */
  const int *neitab;        /* NeiTab(NP,MNEI) */
  const double *fdxe, *fdye;/* FDXE(3,NE), FDYE(3,NE) */
  const double *areas;      /* AREAS(NE) = 2*element area */
  const int *csr_position;  /* CSR_POSITION(NE,3,2) */
  /* nodal attributes */
  const double *tau0var, *evm, *fric, *corif;
  /* boundaries.F / global.F forcing tables */
  const int *nbd;           /* NBD(NETA) */
  const double *amig, *per, *face, *ff;  /* (NBFR) */
  const double *emo, *efa;  /* EMO(NBFR,NETA), EFA(NBFR,NETA) radians */
  const int *nbv, *lbcodei; /* (NVEL) */
  const double *csii, *siii;/* (NVEL) */
  const int *me2gw;         /* (NVELME) */
  const double *bndlen2o3;  /* (NVEL) */
  /* state (in/out) */
  double *eta1, *eta2, *etas;
  double *uu1, *vv1, *uu2, *vv2, *qx1, *qy1, *qx2, *qy2, *h1, *h2;
  double *tk, *tkm;         /* TK(NP), TKM(3,NP) */
  int *nodecode, *nnodecode, *noff, *mju;
  double *totalarea, *alphal;
  double *wsx1, *wsy1, *wsx2, *wsy2, *pr1, *pr2;
  double *coef;             /* COEF(NP,MNEI) */
  double *obccoef;          /* OBCCoef(NETA,MNEI-1) */
  double *gwce_lv, *mom_lv_x, *mom_lv_y;
  const int *nelezng;       /* NEleZNG(NVEL), 1-based (IBTYPE 40 entries) */
  const double *zngif1, *zngif2, *zngif3;
  const int *neitabele;     /* NeiTabEle(NP,MNEI), 1-based, 0 = none */
  const double *barlanht, *barlancfsp;   /* (NVEL) external barriers (IBTYPE 3/13/23) */
  const int *ibconn;        /* (NVEL) internal barriers (IBTYPE 4/24): node across, 1-based */
  const double *barinht, *barincfsb, *barincfsp;   /* (NVEL) */
  const int *nvell;         /* NVELL(NBOU) after closure, barrier segments in pairs */
  const double *pipeht, *pipecoef, *pipediam;   /* (NVEL) pipes of IBTYPE 5/25 barriers */
} orc_arrays_t;

/* Per-step scalars the TIMESTEP driver computes before the hot path. */
typedef struct {
  int it;
  int pad_;
  double timeloc, timeh, rampelev, rampmete, rampextflux, rampintflux;
} orc_step_t;

/* Periodic specified normal flux (same layout as adc_flux_t). */
typedef struct {
  int nffr, flux_settling_it;
  const double *famig, *fper, *fff, *fface, *qnam, *qnph, *enam, *enph;
} orc_flux_t;

/* Non-periodic boundary series, a fort.19 or fort.20 (same layout as
 * adc_series_t): nrec records of NETA (fort.19) or NVEL (fort.20) values. */
typedef struct {
  int nrec, flux_settling_it;
  double interval, start_time;
  const double *values, *values2;
} orc_series_t;

/* Parametric-vortex track (fort.22 fields HollandGet consumes,
 * nws08.F90:827-878) in mesh units; same layout as adc_vortex_fix_t /
 * adc_vortex_t in include/adcgpu.h. */
typedef struct {
  double time, x, y, cpress, vmax, rmw, tvx, tvy;
} orc_vortex_fix_t;

typedef struct {
  int nfix, avg_minute, hemisphere, pad_;
  double start_time, bladj, rho_air, wind_mult, drag_limit;
  const orc_vortex_fix_t *fix;
} orc_vortex_t;

/* Outputs of one step. */
typedef struct {
  int numitr;      /* IPARM(1) returned by JCG */
  int ier;         /* JCG error flag */
  int ncchange;    /* NCCHANGE after wet/dry */
  int status;      /* 0 ok, 1 = non-positive GWCE diagonal (gwce.F:704) */
  double ep;       /* RMS of the GWCE diagonal at the last rebuild */
  double zeta;     /* RPARM(1) after the solve */
  double cme;      /* final eigenvalue estimate RPARM(2) */
  int n_w1_events; /* W1 wetting events that raised TK */
  int pad_;
} orc_stepout_t;

/* ITPACK JCG, same argument list and Fortran conventions as itpackv.F:63. */
void orc_jcg(const int *n, const int *ndim, const int *maxnz, int *jcoef,
             double *coef, double *rhs, double *u, int *iwksp, const int *nw,
             double *wksp, int *iparm, double *rparm, int *ier);
void orc_dfault(int *iparm, double *rparm);
/* Reset the ITPACK module state (the saved q1 flag) to program start. */
void orc_itpack_reset(void);

/* Model-level oracle: owns ITPACK state, IPARM/RPARM, NCChange, EP. */
typedef struct orc_model orc_model;
orc_model *orc_model_create(const orc_params_t *p, orc_arrays_t *a);
void orc_model_destroy(orc_model *m);
/* One TIMESTEP 2DDI subset: shift, friction, GWCE, wet/dry, H2, momentum. */
int orc_model_step(orc_model *m, const orc_step_t *s, orc_stepout_t *out);
/* Individual phases (for phase-level parity tests). */
int orc_model_shift_friction(orc_model *m, const orc_step_t *s);
int orc_model_gwce(orc_model *m, const orc_step_t *s, orc_stepout_t *out);
int orc_model_wetdry(orc_model *m, const orc_step_t *s, orc_stepout_t *out);
int orc_model_momentum(orc_model *m, const orc_step_t *s);
/* NWS = 8 forcing: copies the track; every later step forms WSX2/WSY2/PR2
 * from it after the shift (getMeteorologicalForcing, timestep.F:651).
 * Returns nonzero for an invalid track. */
int orc_model_set_vortex(orc_model *m, const orc_vortex_t *v);
/* The met phase alone (HollandGet + wind.F:1172-1198); nonzero once the
 * run passes the last fix. */
int orc_model_met(orc_model *m, const orc_step_t *s);
/* Specified normal flux (timestep.F:861-880); nonzero without flux boundaries. */
int orc_model_set_flux(orc_model *m, const orc_flux_t *f);
/* fort.19 elevations (NPEBC, gwce.F:1659-1674) and fort.20 fluxes (NFFR <= 0,
 * timestep.F:882-903); nonzero without elevation / flux boundaries.  A run
 * past the last record makes the step return nonzero. */
int orc_model_set_elev_series(orc_model *m, const orc_series_t *s);
int orc_model_set_flux_series(orc_model *m, const orc_series_t *s);
void orc_model_set_ncchange(orc_model *m, int ncchange);
int orc_model_get_ncchange(const orc_model *m);
double orc_model_get_zeta(const orc_model *m);
/* Continue from another implementation's step-to-step state (the module
 * scalars; the arrays come in through the bound orc_arrays_t). */
void orc_model_set_scalars(orc_model *m, int ncchange, double ep, double rparm1, double rparm2,
                           int q1, int vcounter, double vwtratio);

/* Cold-start wet/dry state (cstart.F:1332-1427) and totalAreaCalc
 * (mesh.F:3360-3400): sets NNODECODE, NODECODE, NOFF, ETA2, ETA1, MJU,
 * TotalArea. */
void orc_coldstart(const orc_params_t *p, orc_arrays_t *a);

/* Static mesh and boundary tables (oracle_mesh.cpp, mesh.F), with the
 * argument lists of the library's adc_mesh_* / adc_boundary_setup /
 * adc_coldstart.  0 on success, negative on an invalid mesh. */
int orc_mesh_geometry(int np, int ne, const double *x, const double *y, int *nm,
                      double *fdxe, double *fdye, double *areas);
int orc_mesh_mnei(int np, int ne, const int *nm);
int orc_mesh_neighb(int np, int ne, int mnei, const double *x, const double *y, const int *nm,
                    int *nneigh, int *neitab, int *neimax);
int orc_mesh_csr_positions(int np, int ne, int mnei, const int *nm, const int *neitab,
                           int neimax, int *csr_position);
int orc_boundary_setup(int np, const double *x, const double *y, int nbou, const int *ibtype,
                       const int *seg_ptr, const int *seg_nodes, double costset, int nvel_max,
                       int *nvel_out, int *nbv, int *lbcodei, double *csii, double *siii,
                       int *nvelme_out, int *me2gw, double *bndlen2o3);
int orc_mesh_neitabele(int np, int ne, int mnei, const int *nm, const int *nneigh,
                       const int *neitab, int *neitabele);
int orc_zng_setup(int np, int ne, const double *x, const double *y, const int *nm, int mnei,
                  const int *nneigh, const int *neitab, const double *areas, int nvel,
                  const int *nbv, const int *lbcodei, const double *csii, const double *siii,
                  int *nelezng, double *zngif1, double *zngif2, double *zngif3);
int orc_coldstart_arrays(int np, int ne, int nolifa, double h0, const double *dp, const int *nm,
                         const double *areas, double *eta1, double *eta2, int *nnodecode,
                         int *nodecode, int *noff, int *mju, double *totalarea);

#ifdef __cplusplus
}
#endif
#endif
