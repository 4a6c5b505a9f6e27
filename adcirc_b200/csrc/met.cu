// met.cu -- parametric-vortex met forcing on the device (NWS = 8).
//
// getMeteorologicalForcing (timestep.F:651) for NWS = 8 calls HollandGet
// (nws08.F90:562-717) and turns its 10 m wind and surface pressure into the
// GWCE/momentum forcing WSX2/WSY2/PR2 (wind.F:1172-1198).  Here one thread
// advances the track state (GetHollandStormData, nws08.F90:827-878, whose
// module counter and WTRATIO persist across steps) and every node then
// evaluates the vortex independently.  The step's TimeLoc and RampMete come
// from the device step table, so replayed step graphs need no host work.
//
// The mesh is Cartesian (ICS = 1): the storm centre is in mesh metres, the
// distance is Euclidean and theta = atan2(dy, dx) (thetaLatDep = .false.);
// the reference's DEG2RAD scaling and haversine distance apply to its
// spherical (ICS = 2) input only.  Transcendentals are CUDA's (sqrt, exp,
// pow, sin, cos, atan2).
#include "adc_internal.cuh"

#include <cmath>
#include <cstring>

namespace adc {

constexpr double kE = 2.718281828459045;       // constants.F90:76
constexpr double kOne2Ten = 0.8928;            // constants.F90:105
constexpr double kPrBckgrndMb = 1013.0;        // constants.F90:55
constexpr double kRhoWat0 = 1000.0;            // constants.F90:49

// GetHollandStormData (nws08.F90:827-878) and the per-storm part of
// HollandGet (nws08.F90:602-639).  The position is interpolated with the
// WTRATIO left by the previous call, as the reference does.
__global__ void k_vortex_state(adc_ctx c, const adc_step_t *steps, Flags *flags) {
  griddep_wait();
  VortexState &v = *c.vstate;
  const adc_vortex_fix_t *f = c.vfix;
  const double timeloc = steps[flags->cursor].timeloc;
  int i = v.counter;
  if (timeloc > f[i].time) {
    i = i + 1;
    if (i >= c.vpar.nfix) {   // nws08.F90:847-852: past the end of the track
      v.err = 1;
      flags->status = ADC_ERR_ARG;
      i = c.vpar.nfix - 1;
    }
  }
  const double lon = f[i - 1].x + v.wtratio * (f[i].x - f[i - 1].x);
  const double lat = f[i - 1].y + v.wtratio * (f[i].y - f[i - 1].y);
  v.counter = i;
  if (f[i].cpress < 0.0 || f[i - 1].cpress < 0.0) {
    // a CALM line on either side (nws08.F90:858-872): no storm, WTRATIO kept
    v.calm = 1;
    v.x = lon;
    v.y = lat;
    return;
  }
  v.calm = 0;
  const double wt = (timeloc - f[i - 1].time) / (f[i].time - f[i - 1].time);
  v.wtratio = wt;
  const double cpress = f[i - 1].cpress + wt * (f[i].cpress - f[i - 1].cpress);
  double spd = f[i - 1].vmax + wt * (f[i].vmax - f[i - 1].vmax);
  const double rmw = f[i - 1].rmw + wt * (f[i].rmw - f[i - 1].rmw);
  const double tvx = f[i - 1].tvx + wt * (f[i].tvx - f[i - 1].tvx);
  const double tvy = f[i - 1].tvy + wt * (f[i].tvy - f[i - 1].tvy);
  // HollandGet: pressure deficit floor, translation removal, BL adjustment,
  // the limited Holland B (backgroundWindFac = 1 for the radial-velocity-
  // weighted background model, nws08.F90:480-485)
  double dpdef = kPrBckgrndMb * 100.0 - cpress;
  if (dpdef < 100.0) dpdef = 100.0;
  const double ts = sqrt(tvx * tvx + tvy * tvy);
  spd = spd - 1.0 * ts;
  spd = spd / c.vpar.bladj;
  double b = c.vpar.rho_air * kE * (spd * spd) / dpdef;
  if (b < 1.0) b = 1.0;
  if (b > 2.5) b = 2.5;
  v.x = lon;
  v.y = lat;
  v.cpress = cpress;
  v.dpdef = dpdef;
  v.spd = spd;
  v.b = b;
  v.rmw = rmw * 1000.0;
  v.tvx = tvx;
  v.tvy = tvy;
}

// The node loop of HollandGet (nws08.F90:642-715) followed by the NWS = 8
// stress and pressure of wind.F:1172-1198 (capped Garratt drag,
// wind.F:514-539; no directional reduction, canopy or ice).
__global__ void k_vortex_nodes(adc_ctx c, const adc_step_t *steps, const Flags *flags) {
  griddep_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.np) return;
  const VortexState &v = *c.vstate;
  const double rampmete = steps[flags->cursor].rampmete;
  double wx, wy, prn2;
  if (v.calm) {   // HollandGet's CALM return (nws08.F90:588-601)
    wx = 0.0;
    wy = 0.0;
    prn2 = kPrBckgrndMb * 100.0 / (kRhoWat0 * c.p.g);
  } else {
    const double hemi = c.vpar.hemisphere >= 0 ? 1.0 : -1.0;   // sign(1, lat)
    const double dx = c.x[i] - v.x;
    const double dy = c.y[i] - v.y;
    const double theta = atan2(dy, dx);
    const double rad = sqrt(dx * dx + dy * dy);
    const double f = c.corif[i];
    const double alpha = pow(v.rmw / rad, v.b);
    double press = v.cpress + v.dpdef * exp(-alpha);
    double vr = sqrt(alpha * exp(1.0 - alpha) * v.spd * (v.spd + 0.0) + 0.25 * (rad * rad) * (f * f)) -
                0.5 * rad * fabs(f);
    vr = vr * c.vpar.wind_mult;
    vr = vr * c.vpar.bladj;
    // inflow angle 0 (useInflow = .false.): theta + sign(1,lat)*0 == theta
    wx = (-hemi) * vr * sin(theta + hemi * 0.0);
    wy = hemi * vr * cos(theta + hemi * 0.0);
    // calcTranslationSpeed, radial-velocity-weighted (nws08.F90:746-749)
    const double tsx = (fabs(vr) / v.spd) * v.tvx;
    const double tsy = (fabs(vr) / v.spd) * v.tvy;
    wx = wx + tsx;
    wy = wy + tsy;
    if (c.vpar.avg_minute == 1) {
      wx = wx * kOne2Ten;
      wy = wy * kOne2Ten;
    }
    press = fmax(0.85e5, fmin(1.1e5, press));
    wx = fmax(-200.0, fmin(200.0, wx));
    wy = fmax(-200.0, fmin(200.0, wy));
    prn2 = press / (kRhoWat0 * c.p.g);
  }
  // wind.F:1174-1193
  const double mag = sqrt(wx * wx + wy * wy);
  double drag = 0.001 * (0.75 + 0.067 * mag);
  if (drag > c.vpar.drag_limit) drag = c.vpar.drag_limit;
  const double awr = c.vpar.rho_air / kRhoWat0;   // airwaterdensityrat, wind.F:349
  c.wsx2[i] = rampmete * awr * drag * wx * mag;
  c.wsy2[i] = rampmete * awr * drag * wy * mag;
  const double prdiff = rampmete * (prn2 - c.p.prbckgrnd_mh2o);
  c.pr2[i] = c.p.prbckgrnd_mh2o + prdiff;
}

int launch_met_vortex(adc_ctx *c) {
  if (!c->vortex_on) return ADC_OK;
  launch_k(k_vortex_state, 1, 1, c->stream, *c, c->steps, c->flags);
  launch_k(k_vortex_nodes, nblk(c->np), kThreads, c->stream, *c, c->steps, c->flags);
  c->launches += 2;
  return ADC_OK;
}

// NWS08INIT (nws08.F90:459-477): the first fix pair brackets the start time.
static int vortex_first_pair(const adc_vortex_t *v) {
  const double t = v->start_time;
  for (int i = 1; i < v->nfix; ++i)
    if (std::ceil(t) >= v->fix[i - 1].time && std::floor(t) < v->fix[i].time) return i;
  return -1;
}

}  // namespace adc

using namespace adc;

extern "C" int adc_set_vortex(adc_ctx *c, const adc_vortex_t *v) {
  if (!c || !v || !v->fix || v->nfix < 2) {
    set_error("adc_set_vortex: a track of at least two fixes is required");
    return ADC_ERR_ARG;
  }
  if (c->p.nws == 0) {
    set_error("adc_set_vortex: NWS = 0 in the bound parameters");
    return ADC_ERR_ARG;
  }
  for (int i = 1; i < v->nfix; ++i)
    if (!(v->fix[i].time > v->fix[i - 1].time)) {
      set_error("adc_set_vortex: fix times must increase (fix %d)", i + 1);
      return ADC_ERR_ARG;
    }
  if (!(v->bladj > 0.0) || !(v->rho_air > 0.0)) {
    set_error("adc_set_vortex: BLAdj and rhoAir must be positive");
    return ADC_ERR_ARG;
  }
  const int i0 = vortex_first_pair(v);
  if (i0 < 0) {
    set_error("adc_set_vortex: the track does not cover the start time %g s", v->start_time);
    return ADC_ERR_ARG;
  }
  if (c->vfix) {
    cudaFree(c->vfix);
    c->vfix = nullptr;
  }
  ADC_CUDA(cudaMalloc((void **)&c->vfix, v->nfix * sizeof(adc_vortex_fix_t)));
  ADC_CUDA(cudaMemcpy(c->vfix, v->fix, v->nfix * sizeof(adc_vortex_fix_t), cudaMemcpyHostToDevice));
  if (!c->vstate) ADC_CUDA(cudaMalloc((void **)&c->vstate, sizeof(VortexState)));
  VortexState st;
  memset(&st, 0, sizeof(st));
  st.counter = i0;
  st.wtratio = 1.0;   // module default, nws08.F90:68
  ADC_CUDA(cudaMemcpy(c->vstate, &st, sizeof(st), cudaMemcpyHostToDevice));
  c->vpar = *v;
  c->vpar.fix = nullptr;
  c->vortex_on = 1;
  drop_graphs(c);   // replayed steps must include the forcing
  return ADC_OK;
}
