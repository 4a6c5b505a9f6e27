"""Host-side case assembly: the module arrays ADCIRC_Init would have built.

``build_case`` turns a ``RawMesh`` plus forcing and fort.15-style
parameters into the full set of Fortran-layout arrays bound by
``adc_gpu_bind`` (include/adcgpu.h): mesh tables (mesh.F), boundary tables
(boundaries.F), nodal attributes, tidal forcing tables and the cold-start
state (cstart.F).  ``GpuModel`` wraps the device-resident step API.
"""
from __future__ import annotations

import copy
import ctypes as C
import dataclasses
import math

import numpy as np

from . import _lib
from ._lib import AdcArrays, AdcParams, AdcStep, AdcStepOut, dp_, ip_, ptr

G_DEFAULT = 9.80665          # constants.F90:45
RHOWAT0 = 1000.0             # constants.F90:48
PRBCKGRND_MB = 1013.0        # constants.F90:55

STATE_F64 = ("eta1", "eta2", "etas", "uu1", "vv1", "uu2", "vv2", "qx1", "qy1", "qx2", "qy2",
             "h1", "h2", "tk", "tkm", "totalarea", "alphal", "wsx1", "wsy1", "wsx2", "wsy2",
             "pr1", "pr2", "coef", "obccoef", "gwce_lv", "mom_lv_x", "mom_lv_y")
STATE_I32 = ("nodecode", "nnodecode", "noff", "mju")


@dataclasses.dataclass
class Schedule:
    """TIMESTEP time and ramp bookkeeping (timestep.F:257-353)."""
    dt: float
    statim: float = 0.0      # days
    reftim: float = 0.0      # days
    nramp: int = 1
    dramp: float = 0.5       # days (elevation ramp, DRampElev)
    dramp_mete: float = 0.5  # days
    dunramp_mete: float = 0.0
    dramp_extflux: float | None = None   # days; None: the elevation ramp's
    dramp_intflux: float | None = None   # days (barrier overflow); None: the elevation ramp's
    flux_settling_time: float = 0.0      # days (fort.15 FluxSettlingTime, NRAMP >= 2)

    @property
    def flux_settling_it(self) -> int:
        """FluxSettlingIT, timestep.F:243-245."""
        return int(self.flux_settling_time * 86400.0 / self.dt)

    def step(self, it: int) -> AdcStep:
        timeloc = it * self.dt + self.statim * 86400.0
        timeh = it * self.dt + (self.statim - self.reftim) * 86400.0
        if self.nramp == 0:
            relev = rmete = 1.0
        else:
            relev = math.tanh((2.0 * timeloc / 86400.0) / self.dramp)
            rmete = math.tanh((2.0 * (timeloc / 86400.0 - self.dunramp_mete)) / self.dramp_mete)
        dix = self.dramp if self.dramp_intflux is None else self.dramp_intflux
        if self.nramp == 0:
            rint = 1.0
        else:
            rint = math.tanh((2.0 * timeloc / 86400.0) / dix)
        fsit = self.flux_settling_it
        if self.nramp > 1 and fsit > 0:
            # every forcing but the river flux waits for the flux to settle,
            # then ramps from there (timestep.F:314-345)
            if it < fsit + 10:
                relev = rmete = rint = 0.0
            else:
                tl = (it - fsit - 10) * self.dt + self.statim * 86400.0
                relev = math.tanh((2.0 * tl / 86400.0) / self.dramp)
                rint = math.tanh((2.0 * tl / 86400.0) / dix)
                if self.nramp != 8:
                    rmete = math.tanh((2.0 * tl / 86400.0) / self.dramp_mete)
        if self.dramp < 1.0e-6:
            relev = 1.0
        if self.dramp_mete < 1.0e-6:
            rmete = 1.0
        if dix < 1.0e-6:
            rint = 1.0
        s = AdcStep()
        s.it = it
        s.timeloc = timeloc
        s.timeh = timeh
        s.rampelev = relev
        s.rampmete = rmete
        dfx = self.dramp if self.dramp_extflux is None else self.dramp_extflux
        if self.nramp == 0 or dfx < 1.0e-6:
            s.rampextflux = 1.0
        else:
            s.rampextflux = math.tanh((2.0 * timeloc / 86400.0) / dfx)
        s.rampintflux = rint
        return s

    def steps(self, it0: int, n: int):
        arr = (AdcStep * n)()
        for k in range(n):
            arr[k] = self.step(it0 + k)
        return arr


@dataclasses.dataclass
class Case:
    name: str
    params: dict
    sizes: dict
    arrays: dict                 # name -> numpy array (Fortran layout)
    schedule: Schedule
    meta: dict = dataclasses.field(default_factory=dict)
    vortex: "Vortex | None" = None   # NWS = 8 parametric-vortex track
    flux: "Flux | None" = None       # specified normal flux (IBTYPE 2/12/22)
    elev_series: "Series | None" = None   # non-periodic boundary elevations (fort.19)
    flux_series: "Series | None" = None   # non-periodic normal fluxes (fort.20, NFFR <= 0)

    def clone(self) -> "Case":
        c = copy.copy(self)
        c.arrays = {k: v.copy(order="F") for k, v in self.arrays.items()}
        c.params = dict(self.params)
        return c

    def params_struct(self) -> AdcParams:
        p = AdcParams()
        for k, v in self.params.items():
            setattr(p, k, v)
        return p

    def arrays_struct(self) -> AdcArrays:
        a = AdcArrays()
        for k in ("np", "ne", "mnei", "neta", "nbfr", "nvel", "nvelme", "nbou"):
            setattr(a, k, int(self.sizes[k]))
        for name, typ in _lib.ARRAY_FIELDS:
            arr = self.arrays[name]
            want = np.int32 if typ is ip_ else np.float64
            assert arr.dtype == want and arr.flags.f_contiguous, name
            setattr(a, name, ptr(arr, typ))
        return a

    def state(self):
        return {k: self.arrays[k] for k in STATE_F64 + STATE_I32}


@dataclasses.dataclass
class Flux:
    """Periodic specified normal flux on the flux boundaries (IBTYPE 2, 12,
    22, 32, 52): constituents (rad/s, s, nodal factor, rad) and per boundary
    entry (NVEL) amplitudes [m^2/s] and phases [rad], zero off flux entries;
    flux_settling_it is FluxSettlingIT (river radiation, IBTYPE 52)."""
    famig: np.ndarray
    fper: np.ndarray
    fff: np.ndarray
    fface: np.ndarray
    qnam: np.ndarray   # (NFFR, NVEL)
    qnph: np.ndarray   # (NFFR, NVEL)
    flux_settling_it: int = 0
    enam: "np.ndarray | None" = None   # (NFFR, NVEL) elevation constituents (IBTYPE 32)
    enph: "np.ndarray | None" = None

    def struct(self, cls=None):
        """(struct, backing arrays); keep both alive while in use."""
        cls = cls or _lib.AdcFlux
        keep = [np.ascontiguousarray(a, np.float64) for a in (self.famig, self.fper, self.fff,
                                                                self.fface)]
        keep += [np.asfortranarray(a, np.float64) for a in (self.qnam, self.qnph)]
        names = ["famig", "fper", "fff", "fface", "qnam", "qnph"]
        if self.enam is not None:
            keep += [np.asfortranarray(a, np.float64) for a in (self.enam, self.enph)]
            names += ["enam", "enph"]
        f = cls()
        f.nffr = int(keep[0].size)
        f.flux_settling_it = int(self.flux_settling_it)
        for name, a in zip(names, keep):
            setattr(f, name, a.ctypes.data_as(dp_))
        return f, keep


@dataclasses.dataclass
class Series:
    """A non-periodic boundary time series: the records of a fort.19
    (`values` (nrec, NETA) boundary elevations [m]) or of a fort.20
    (`values` (nrec, NVEL) normal fluxes [m^2/s], zero off the entries of
    code 2/12/22/32, and `values2` the elevations of code-32 entries), one
    record every `interval` seconds from `start_time` (STATIM*86400).
    `flux_settling_it` is FluxSettlingIT for a fort.20 with river-radiation
    entries."""
    interval: float
    values: np.ndarray
    values2: "np.ndarray | None" = None
    start_time: float = 0.0
    flux_settling_it: int = 0

    def struct(self, cls=None):
        """(struct, backing arrays); keep both alive while in use."""
        cls = cls or _lib.AdcSeries
        keep = [np.ascontiguousarray(self.values, np.float64)]
        if self.values2 is not None:
            keep.append(np.ascontiguousarray(self.values2, np.float64))
            assert keep[1].shape == keep[0].shape
        s = cls()
        s.nrec = int(keep[0].shape[0])
        s.flux_settling_it = int(self.flux_settling_it)
        s.interval, s.start_time = float(self.interval), float(self.start_time)
        s.values = keep[0].ctypes.data_as(dp_)
        if len(keep) > 1:
            s.values2 = keep[1].ctypes.data_as(dp_)
        return s, keep


@dataclasses.dataclass
class Vortex:
    """A parametric-vortex track in mesh coordinates (fort.22 for NWS = 8).

    fixes: (n, 8) float64 rows of (time [s], x [m], y [m], central pressure
    [Pa], Vmax [m/s, 10 m], RMW [km], TVX, TVY [m/s]).
    """
    fixes: np.ndarray
    start_time: float = 0.0
    avg_minute: int = 1
    hemisphere: int = 1
    bladj: float = 0.9
    rho_air: float = 1.293        # constants.F90 default rhoAir
    wind_mult: float = 1.0
    drag_limit: float = 0.0035    # wind.F default WindDragLimit

    def struct(self):
        """(AdcVortex, backing fix array); keep both alive while in use."""
        fx = np.ascontiguousarray(self.fixes, dtype=np.float64)
        arr = (_lib.AdcVortexFix * len(fx))()
        for k, row in enumerate(fx):
            arr[k] = _lib.AdcVortexFix(*[float(v) for v in row])
        v = _lib.AdcVortex()
        v.nfix, v.avg_minute, v.hemisphere = len(fx), self.avg_minute, self.hemisphere
        v.start_time, v.bladj, v.rho_air = self.start_time, self.bladj, self.rho_air
        v.wind_mult, v.drag_limit = self.wind_mult, self.drag_limit
        v.fix = C.cast(arr, C.POINTER(_lib.AdcVortexFix))
        return v, arr


def straight_track(x0: float, y0: float, heading_deg: float, speed: float, pc_hpa: float,
                   rmw_km: float, holland_b: float, hours: float, interval_h: float = 6.0,
                   bladj: float = 0.9, rho_air: float = 1.293) -> Vortex:
    """Straight constant-speed track whose limited Holland B equals
    `holland_b`: Vmax is chosen so that HollandGet's B = rhoAir*e*spd^2/dp
    (nws08.F90:631) reproduces it after the translation removal and the
    boundary-layer adjustment (nws08.F90:621-627)."""
    dp = PRBCKGRND_MB * 100.0 - pc_hpa * 100.0
    spd_bl = math.sqrt(holland_b * dp / (rho_air * math.e))
    vmax = spd_bl * bladj + speed
    h = math.radians(heading_deg)
    tvx, tvy = speed * math.cos(h), speed * math.sin(h)
    n = int(math.ceil(hours / interval_h)) + 1
    rows = []
    for k in range(n):
        t = k * interval_h * 3600.0
        rows.append((t, x0 + tvx * t, y0 + tvy * t, pc_hpa * 100.0, vmax, rmw_km, tvx, tvy))
    return Vortex(np.array(rows), bladj=bladj, rho_air=rho_air)


def default_params(dt: float, **kw) -> dict:
    p = dict(dt=dt, g=G_DEFAULT, a00=0.35, b00=0.30, c00=0.35, h0=0.05, velmin=0.01,
             slim=1.0e9, hbreak=1.0, ftheta=1.0, fgamma=1.0, convcr=1.0e-10,
             prbckgrnd_mh2o=100.0 * PRBCKGRND_MB / (RHOWAT0 * G_DEFAULT),
             ifnlfa=1, ifnlct=1, ifnlcat=1, nolifa=2, iflinbf=0, ifnlbf=1, ifhybf=0,
             itmax=200, nws=0, ifwind=1, isldia=0, pad_=0)
    p.update(kw)
    return p


def _f(a, dtype):
    return np.asfortranarray(np.asarray(a, dtype=dtype))


def tau0_nodal(scheme: float, depth: np.ndarray) -> np.ndarray:
    """Tau0Var for a negative fort.15 TAU0 (nodalattr.F:1872-1876 via
    Tau0NodalValue, nodalattr.F:2084-2100): -2 varies smoothly with depth
    (0.005 below 200 m, 1/depth from 200 m to 1 m, 1 above), any other
    negative value switches from 0.005 to 0.020 at 10 m depth."""
    d = np.asarray(depth, np.float64)
    if scheme == -2.0:
        out = np.where(d >= 200.0, np.float64(np.float32(0.005)), 0.0)   # REAL literal 0.005
        mid = (d < 200.0) & (d >= 1.0)
        out[mid] = np.float64(np.float32(1.0)) / d[mid]
        out[d < 1.0] = 1.0
        return out
    return np.where(d <= 10.0, 0.020, 0.005)


@dataclasses.dataclass
class MeshPrep:
    """The one-time table builders build_case calls, each with the argument
    list of the library's adc_mesh_geometry, adc_mesh_mnei, adc_mesh_neighb,
    adc_mesh_csr_positions, adc_boundary_setup and adc_coldstart (0 on
    success).  `product_prep()` gives the library's own."""
    geometry: object
    mnei: object
    neighb: object
    csr_positions: object
    boundary_setup: object
    coldstart: object
    zng_setup: object = None
    neitabele: object = None


def product_prep() -> MeshPrep:
    lib = _lib.load()
    return MeshPrep(lib.adc_mesh_geometry, lib.adc_mesh_mnei, lib.adc_mesh_neighb,
                    lib.adc_mesh_csr_positions, lib.adc_boundary_setup, lib.adc_coldstart,
                    lib.adc_zng_setup, lib.adc_mesh_neitabele)


def build_case(raw, params: dict, schedule: Schedule, tides, cf: float = 0.0025,
               tau0: float = 0.005, eslm: float = 5.0, cori: float = 1.0e-4,
               anginn: float = 110.0, eta0=None, prep: MeshPrep | None = None) -> Case:
    """Assemble every array the hot path binds.

    tides: list of (amig [rad/s], face [rad], ff, emo (NETA,), efa (NETA,) [rad])
    prep: the table builders (default: the library's, `product_prep()`).
    """
    lib = prep if prep is not None else product_prep()
    npn = int(raw.x.size)
    ne = int(raw.nm.shape[0])
    x = _f(raw.x, np.float64)
    y = _f(raw.y, np.float64)
    dp = _f(raw.dp, np.float64)
    nm = _f(raw.nm + 1, np.int32)                      # NM(NE,3)
    fdxe = np.zeros((3, ne), np.float64, order="F")
    fdye = np.zeros((3, ne), np.float64, order="F")
    areas = np.zeros(ne, np.float64)
    rc = lib.geometry(npn, ne, ptr(x, dp_), ptr(y, dp_), ptr(nm, ip_), ptr(fdxe, dp_),
                               ptr(fdye, dp_), ptr(areas, dp_))
    if rc != 0:
        raise RuntimeError(f"adc_mesh_geometry failed: {rc}")
    mnei = lib.mnei(npn, ne, ptr(nm, ip_))
    if mnei < 3:
        raise RuntimeError(f"adc_mesh_mnei failed: {mnei}")
    nneigh = np.zeros(npn, np.int32)
    neitab = np.zeros((npn, mnei), np.int32, order="F")
    neimax = C.c_int(0)
    rc = lib.neighb(npn, ne, mnei, ptr(x, dp_), ptr(y, dp_), ptr(nm, ip_),
                             ptr(nneigh, ip_), ptr(neitab, ip_), C.byref(neimax))
    if rc != 0:
        raise RuntimeError(f"adc_mesh_neighb failed: {rc}")
    csr = np.zeros((ne, 3, 2), np.int32, order="F")
    rc = lib.csr_positions(npn, ne, mnei, ptr(nm, ip_), ptr(neitab, ip_),
                                    neimax.value, ptr(csr, ip_))
    if rc != 0:
        raise RuntimeError(f"adc_mesh_csr_positions failed: {rc}")
    # boundaries
    nbd = _f(raw.open_nodes + 1, np.int32)
    neta = int(nbd.size)
    # an internal barrier (IBTYPE 4/24) is set up as its front face and then
    # its back face, reversed (mesh.F:2158-2192)
    faces = []
    for k, (t, s) in enumerate(raw.land_segments):
        if t in (4, 24, 5, 25):
            back = np.asarray(raw.barriers[k][3], np.int64)
            faces += [(t, np.asarray(s, np.int64)), (t, back[::-1])]
        else:
            faces.append((t, np.asarray(s, np.int64)))
    ibtype = np.array([t for t, _ in faces], np.int32)
    segs = [s + 1 for _, s in faces]
    seg_ptr = np.zeros(len(segs) + 1, np.int32)
    seg_ptr[1:] = np.cumsum([s.size for s in segs])
    seg_nodes = np.concatenate(segs).astype(np.int32)
    nvel_max = int(seg_nodes.size + len(segs) + 1)
    nbv = np.zeros(nvel_max, np.int32)
    lbc = np.zeros(nvel_max, np.int32)
    csii = np.zeros(nvel_max, np.float64)
    siii = np.zeros(nvel_max, np.float64)
    me2gw = np.zeros(nvel_max, np.int32)
    bndlen = np.zeros(nvel_max, np.float64)
    nvel = C.c_int(0)
    nvelme = C.c_int(0)
    rc = lib.boundary_setup(npn, ptr(x, dp_), ptr(y, dp_), len(segs), ptr(ibtype, ip_),
                                ptr(seg_ptr, ip_), ptr(seg_nodes, ip_),
                                math.cos(anginn * math.pi / 180.0), nvel_max, C.byref(nvel),
                                ptr(nbv, ip_), ptr(lbc, ip_), ptr(csii, dp_), ptr(siii, dp_),
                                C.byref(nvelme), ptr(me2gw, ip_), ptr(bndlen, dp_))
    if rc != 0:
        raise RuntimeError(f"adc_boundary_setup failed: {rc}")
    nv, nme = nvel.value, nvelme.value
    # NeiTabEle (used by the Galerkin zero-gradient entries, IBTYPE 41)
    neitabele = np.zeros((npn, mnei), np.int32, order="F")
    if lib.neitabele is not None:
        rc = lib.neitabele(npn, ne, mnei, ptr(nm, ip_), ptr(nneigh, ip_), ptr(neitab, ip_),
                           ptr(neitabele, ip_))
        if rc != 0:
            raise RuntimeError(f"NeiTabEle failed: {rc}")
    # zero-normal-gradient fictitious nodes (IBTYPE 40), mesh.F:2434-2512
    nvz = max(nv, 1)
    nelezng = np.zeros(nvz, np.int32)
    zngif = [np.zeros(nvz) for _ in range(3)]
    if (lbc[:nv] == 40).any():
        if lib.zng_setup is None:
            raise RuntimeError("the table builders have no zero-normal-gradient setup")
        rc = lib.zng_setup(npn, ne, ptr(x, dp_), ptr(y, dp_), ptr(nm, ip_), mnei, ptr(nneigh, ip_),
                           ptr(neitab, ip_), ptr(areas, dp_), nv, ptr(nbv, ip_), ptr(lbc, ip_),
                           ptr(csii, dp_), ptr(siii, dp_), ptr(nelezng, ip_), ptr(zngif[0], dp_),
                           ptr(zngif[1], dp_), ptr(zngif[2], dp_))
        if rc != 0:
            raise RuntimeError(f"zero-normal-gradient setup failed: {rc}")
    # barriers per entry, in the entry order of the boundary setup (islands
    # gain a closing node; internal barriers give two faces), and NVELL as
    # mesh.F leaves it (closed islands, barrier pairs)
    barlanht, barlancfsp = np.zeros(max(nv, 1)), np.zeros(max(nv, 1))
    ibconn = np.zeros(max(nv, 1), np.int32)
    barin = [np.zeros(max(nv, 1)) for _ in range(3)]
    pipes = [np.zeros(max(nv, 1)) for _ in range(3)]
    nvell = np.zeros(max(len(raw.land_segments), 1), np.int32)
    j = 0
    for k, (t, nodes) in enumerate(raw.land_segments):
        n = len(nodes)
        if t in (1, 11, 21) and nodes[0] != nodes[-1]:
            n += 1
        nvell[k] = n
        if t in (3, 13, 23):
            barlanht[j:j + n], barlancfsp[j:j + n] = raw.barriers[k]
        if t in (4, 24, 5, 25):
            vals = [np.asarray(v) for v in raw.barriers[k]]
            back = vals[3]
            front = np.asarray(nodes, np.int64)
            ibconn[j:j + n] = back + 1
            ibconn[j + n:j + 2 * n] = front[::-1] + 1
            per_entry = list(zip(barin, vals[:3]))
            if t in (5, 25):
                per_entry += list(zip(pipes, vals[4:7]))
            for arr, v in per_entry:
                arr[j:j + n] = v
                arr[j + n:j + 2 * n] = v[::-1]
            n *= 2
        j += n
    if j != nv:
        raise RuntimeError(f"boundary entries {j} != NVEL {nv}")
    nbfr = len(tides)
    amig = _f([t[0] for t in tides], np.float64)
    face = _f([t[1] for t in tides], np.float64)
    ff = _f([t[2] for t in tides], np.float64)
    per = _f([2.0 * math.pi / t[0] if t[0] != 0 else 0.0 for t in tides], np.float64)
    emo = np.zeros((max(nbfr, 1), max(neta, 1)), np.float64, order="F")
    efa = np.zeros((max(nbfr, 1), max(neta, 1)), np.float64, order="F")
    for j, t in enumerate(tides):
        emo[j, :neta] = t[3]
        efa[j, :neta] = t[4]
    A = dict(
        x=x, y=y, dp=dp, nm=nm, nneigh=nneigh, neitab=neitab, fdxe=fdxe, fdye=fdye,
        areas=areas, csr_position=csr,
        tau0var=np.full(npn, tau0) if tau0 >= 0.0 else tau0_nodal(tau0, dp),
        evm=np.full(npn, eslm), fric=np.full(npn, cf),
        corif=np.full(npn, cori),
        nbd=nbd, amig=amig if nbfr else _f([0.0], np.float64),
        per=per if nbfr else _f([0.0], np.float64),
        face=face if nbfr else _f([0.0], np.float64),
        ff=ff if nbfr else _f([0.0], np.float64), emo=emo, efa=efa,
        nbv=_f(nbv[:max(nv, 1)], np.int32), lbcodei=_f(lbc[:max(nv, 1)], np.int32),
        csii=_f(csii[:max(nv, 1)], np.float64), siii=_f(siii[:max(nv, 1)], np.float64),
        me2gw=_f(me2gw[:max(nme, 1)], np.int32),
        bndlen2o3=_f(bndlen[:max(nv, 1)], np.float64),
        nelezng=nelezng, zngif1=zngif[0], zngif2=zngif[1], zngif3=zngif[2], neitabele=neitabele,
        barlanht=barlanht, barlancfsp=barlancfsp, ibconn=ibconn, barinht=barin[0],
        barincfsb=barin[1], barincfsp=barin[2], nvell=nvell,
        pipeht=pipes[0], pipecoef=pipes[1], pipediam=pipes[2],
    )
    for k in STATE_F64:
        A[k] = np.zeros(npn, np.float64)
    A["tkm"] = np.zeros((3, npn), np.float64, order="F")
    A["alphal"] = np.ones(ne, np.float64)
    A["coef"] = np.zeros((npn, mnei), np.float64, order="F")
    A["obccoef"] = np.zeros((max(neta, 1), mnei - 1), np.float64, order="F")
    for k in STATE_I32:
        A[k] = np.zeros(npn, np.int32)
    A["noff"] = np.ones(ne, np.int32)
    prb = params["prbckgrnd_mh2o"]
    A["pr1"][:] = prb
    A["pr2"][:] = prb
    if eta0 is not None:
        A["eta2"][:] = eta0
    rc = lib.coldstart(npn, ne, params["nolifa"], params["h0"], ptr(dp, dp_), ptr(nm, ip_),
                           ptr(areas, dp_), ptr(A["eta1"], dp_), ptr(A["eta2"], dp_),
                           ptr(A["nnodecode"], ip_), ptr(A["nodecode"], ip_), ptr(A["noff"], ip_),
                           ptr(A["mju"], ip_), ptr(A["totalarea"], dp_))
    if rc != 0:
        raise RuntimeError(f"adc_coldstart failed: {rc}")
    for k, v in A.items():
        if not v.flags.f_contiguous:
            A[k] = np.asfortranarray(v)
    sizes = dict(np=npn, ne=ne, mnei=mnei, neta=neta, nbfr=nbfr, nvel=nv, nvelme=nme,
                 nbou=len(raw.land_segments), neimax=neimax.value)
    meta = dict(raw.meta)
    meta["build"] = dict(cf=cf, tau0=tau0, eslm=eslm, cori=cori, anginn=anginn)
    meta["raw"] = raw            # the mesh as built (write it with adcirc_io.write_fort14)
    return Case(raw.name, dict(params), sizes, A, schedule, meta)


# --------------------------------------------------------------------------
# Cases from ADCIRC input files, and input files from cases
# --------------------------------------------------------------------------

def _raw_lbcodes(raw) -> np.ndarray:
    """IBTYPE of every flux-boundary node of a RawMesh in fort.14 order:
    the flux records of a fort.15 follow it (island closure nodes carry no
    record)."""
    if not raw.land_segments:
        return np.zeros(0, np.int32)
    return np.concatenate([np.full(len(nodes), t, np.int32) for t, nodes in raw.land_segments])


def case_from_files(fort14, fort15, vortex: "Vortex | None" = None,
                    prep: MeshPrep | None = None, fort19=None, fort20=None, fort22=None) -> Case:
    """A Case from a fort.14 mesh and a fort.15 parameter file, with the
    parameter derivations of the reference: IFNLFA/IFNLCT/IFNLCAT from
    NOLIFA/NOLICA/NOLICAT (adcirc.F:287-290, 376-384), the friction flags
    and FRIC = CF (or TAU when NOLIBF = 0) (nodalattr.F:1974-2001), the ramps
    of NRAMP (read_input.F:2893-2955), periodic elevation constituents and,
    with flux boundaries, the periodic flux constituents.  As the reference
    does, a fort.19 beside the fort.15 adds non-periodic boundary
    elevations (read_input.F:1893-1898), NFFR <= 0 reads the fluxes from
    the fort.20 and NWS = 8 the track from the fort.22 (unless `vortex` is
    given); `fort19`/`fort20`/`fort22` name other paths.  Runs this path
    does not cover raise NotImplementedError: ICS = 2, NCOR = 1, tidal
    potential, hot starts and TAU0 = -5."""
    import pathlib
    from . import adcirc_io
    here = pathlib.Path(fort15).parent
    side = lambda given, name: pathlib.Path(given) if given is not None else here / name
    raw = adcirc_io.read_fort14(fort14)
    neta = int(raw.open_nodes.size)
    f = adcirc_io.read_fort15(fort15, neta, _raw_lbcodes(raw))
    why = []
    if f.ics != 1:
        why.append("ICS = 2 (spherical coordinates)")
    if f.ncor != 0:
        why.append("NCOR = 1 (latitude-dependent Coriolis)")
    if f.ntip != 0:
        why.append("NTIP > 0 (tidal potential)")
    if f.ihot != 0:
        why.append("IHOT > 0 (use adc_hotstart_read)")
    if f.tau0 == -5.0:
        why.append("TAU0 = -5 (time-varying TAU0)")
    has_flux = any(t in (2, 12, 22, 52, 32) for t, _ in raw.land_segments)
    if has_flux and f.nffr <= 0 and not side(fort20, "fort.20").exists():
        why.append("NFFR <= 0 without a fort.20")
    if abs(f.nws) == 8 and vortex is None and not side(fort22, "fort.22").exists():
        why.append("NWS = 8 without a fort.22 track")
    if why:
        raise NotImplementedError(f"{fort15}: " + "; ".join(why))
    params = default_params(
        f.dtdp, g=f.g, a00=f.a00, b00=f.b00, c00=f.c00, h0=f.h0, slim=f.slim, convcr=f.convcr,
        itmax=f.itmax, isldia=f.isldia, nolifa=f.nolifa, ifnlfa=int(f.nolifa != 0),
        ifnlct=int(f.nolica != 0), ifnlcat=int(f.nolicat != 0),
        iflinbf=int(f.nolibf == 0), ifnlbf=int(f.nolibf in (1, 3)), ifhybf=int(f.nolibf == 2),
        nws=int(abs(f.nws)))
    if f.nolifa == 2:
        params["velmin"] = f.velmin
    if f.nolibf in (2, 3):
        params.update(hbreak=f.hbreak, ftheta=f.ftheta)
    if f.nolibf == 2:
        params["fgamma"] = f.fgamma
    sched = Schedule(dt=f.dtdp, statim=f.statim, reftim=f.reftim, nramp=f.nramp, dramp=f.dramp_elev,
                     dramp_mete=f.dramp_mete, dunramp_mete=f.dunramp_mete,
                     dramp_extflux=f.dramp_extflux, dramp_intflux=f.dramp_intflux,
                     flux_settling_time=f.flux_settling_time)
    tides = [(float(f.amig[k]), float(f.face[k]), float(f.ff[k]), f.emo[k].copy(), f.efa[k].copy())
             for k in range(f.nbfr)]
    case = build_case(raw, params, sched, tides, cf=f.tau if f.nolibf == 0 else f.cf, tau0=f.tau0,
                      eslm=f.eslm, cori=f.cori, anginn=f.anginn, prep=prep)
    if f.nffr > 0:
        lbc = case.arrays["lbcodei"][:case.sizes["nvel"]]
        f = adcirc_io.read_fort15(fort15, neta, lbc)      # flux records on the case's NVEL order
        fper = np.where(f.famig != 0.0, 2.0 * math.pi / np.where(f.famig != 0.0, f.famig, 1.0), 0.0)
        has32 = (lbc == 32).any()
        case.flux = Flux(f.famig.copy(), fper, f.fff.copy(), f.fface.copy(), f.qnam.copy(),
                         f.qnph.copy(), flux_settling_it=sched.flux_settling_it,
                         enam=f.enam.copy() if has32 else None, enph=f.enph.copy() if has32 else None)
    lbc = case.arrays["lbcodei"][:case.sizes["nvel"]]
    start = f.statim * 86400.0
    p19 = side(fort19, "fort.19")
    if neta > 0 and p19.exists():
        case.elev_series = adcirc_io.read_fort19(p19, neta, start_time=start)
    if has_flux and f.nffr <= 0:
        case.flux_series = adcirc_io.read_fort20(side(fort20, "fort.20"), lbc, start_time=start,
                                                 flux_settling_it=sched.flux_settling_it)
    if abs(f.nws) == 8:
        if vortex is None:
            vortex = adcirc_io.read_fort22(side(fort22, "fort.22"), f.irefyr, f.irefmo, f.irefday,
                                           f.irefhr, f.slam0, f.sfea0, f.rnday, bladj=f.bladj,
                                           start_time=start, drag_limit=f.wind_drag_limit,
                                           avg_minute=f.windspeed_averaging_minute,
                                           wind_mult=f.wind_multiplier)
        case.vortex = vortex
    case.meta["fort15"] = f
    return case


def apply_hotstart(case: Case, hs: dict) -> int:
    """Loads a reference hotstart (adcirc_io.read_fort67) into a case's
    arrays as hstart.F does (:511-533, 764-768): ETA1, ETA2, UU2, VV2, NOFF,
    NNODECODE and NODECODE from the file, then H1 = DP + IFNLFA ETA1,
    H2 = DP + IFNLFA ETA2, ETAS = ETA2 - ETA1, QX2 = UU2 H2, QY2 = VV2 H2.
    A vortex track is repositioned to the file's time (NWS08INIT picks the
    fix pair from TimeLoc) and non-periodic series are advanced as
    hstart.F:857-883 advances them.  Returns ITHS; the run continues with
    step ITHS + 1.  Not carried over, because the reference recomputes them
    at start-up rather than reading them: the met fields at ITHS
    (hotstartMeteorologicalForcing, hstart.F:1442) and the flux history QN1,
    QN2 of fort.20 boundaries (hstart.F:949-971); the first step after the
    load starts them from the background pressure, no wind and zero flux."""
    a = case.arrays
    if hs["eta1"].size != case.sizes["np"] or hs["noff"].size != case.sizes["ne"]:
        raise ValueError("the hotstart file holds another mesh")
    ifnlfa = case.params["ifnlfa"]
    for k in ("eta1", "eta2", "uu2", "vv2"):
        a[k][:] = hs[k]
    a["noff"][:] = hs["noff"]
    a["nnodecode"][:] = hs["nodecode"]
    a["nodecode"][:] = hs["nodecode"]
    a["h1"][:] = a["dp"] + ifnlfa * a["eta1"]
    a["h2"][:] = a["dp"] + ifnlfa * a["eta2"]
    a["etas"][:] = a["eta2"] - a["eta1"]
    a["qx2"][:] = a["uu2"] * a["h2"]
    a["qy2"][:] = a["vv2"] * a["h2"]
    iths, timeloc = int(hs["it"]), float(hs["timeloc"])
    if case.vortex is not None:
        case.vortex = dataclasses.replace(case.vortex, start_time=timeloc)
    for attr in ("elev_series", "flux_series"):
        ser = getattr(case, attr)
        if ser is not None:
            setattr(case, attr, series_at_hotstart(ser, iths, timeloc, case.schedule))
    return iths


def series_at_hotstart(ser: Series, iths: int, timeloc: float, sched: Schedule) -> Series:
    """The record pair a reference run holds after a hotstart at step ITHS
    (hstart.F:857-883: the read-ahead replayed over steps 1 .. ITHS-1, then
    once more for TimeLoc), as a series that starts there."""
    t1 = ser.start_time
    t2 = t1 + ser.interval
    k = 0
    for it in range(1, iths):
        timeit = it * sched.dt + sched.statim * 86400.0
        if timeit > t2:
            t1 = t2
            t2 = t1 + ser.interval
            k += 1
    if timeloc > t2:
        t1 = t2
        k += 1
    if k + 2 > ser.values.shape[0]:
        raise ValueError("the series ends before the hotstart time")
    v2 = None if ser.values2 is None else ser.values2[k:]
    return dataclasses.replace(ser, values=ser.values[k:], values2=v2, start_time=t1)


def fort15_for_case(case: Case, rnday: float = 1.0, rundes: str = "", runid: str = "run"):
    """The fort.15 values of a Case (the inverse of case_from_files), for
    adcirc_io.write_fort15: NRAMP 8 carries the case's separate elevation,
    flux and met ramps; outputs, stations and harmonic analysis are off."""
    from . import adcirc_io
    p, b, s = case.params, case.meta.get("build", {}), case.schedule
    o = _lib.AdcFort15()
    o.rundes = (rundes or case.name).encode()[:80]
    o.runid = runid.encode()[:80]
    o.nfover, o.nabout, o.nscreen, o.ihot, o.ics, o.im = 1, 1, 0, 0, 1, 0
    o.nolibf = 0 if p["iflinbf"] else (2 if p["ifhybf"] else 1)
    o.nolifa, o.nolica, o.nolicat = p["nolifa"], p["ifnlct"], p["ifnlcat"]
    o.ncor, o.ntip, o.nws = 0, 0, p["nws"]
    o.g, o.tau0, o.dtdp, o.statim, o.reftim, o.rnday = p["g"], b.get("tau0", 0.005), p["dt"], \
        s.statim, s.reftim, rnday
    if o.nws:
        o.irefyr, o.irefmo, o.irefday, o.irefhr, o.storm_number = 2000, 1, 1, 0, 1
        o.bladj = case.vortex.bladj if case.vortex is not None else 0.9
    o.nramp = 0 if s.nramp == 0 else 8
    o.dramp = o.dramp_elev = o.dramp_tip = o.dramp_wrad = s.dramp
    o.dramp_intflux = s.dramp if s.dramp_intflux is None else s.dramp_intflux
    o.dramp_extflux = s.dramp if s.dramp_extflux is None else s.dramp_extflux
    o.flux_settling_time = s.flux_settling_time
    o.dramp_mete, o.dunramp_mete = s.dramp_mete, s.dunramp_mete
    o.a00, o.b00, o.c00, o.h0, o.velmin = p["a00"], p["b00"], p["c00"], p["h0"], p["velmin"]
    o.nodedrymin, o.nodewetmin = 0, 0
    cf = b.get("cf", 0.0025)
    o.tau, o.cf = cf, cf
    o.hbreak, o.ftheta, o.fgamma = p["hbreak"], p["ftheta"], p["fgamma"]
    o.eslm, o.cori, o.anginn = b.get("eslm", 5.0), b.get("cori", 1.0e-4), b.get("anginn", 110.0)
    o.convcr, o.itmax, o.ititer, o.isldia = p["convcr"], p["itmax"], 1, p["isldia"]
    o.slim, o.has_slim = p["slim"], int(p["slim"] != 1.0e9)
    o.wind_drag_limit = case.vortex.drag_limit if case.vortex is not None else 0.0035
    o.has_wind_drag_limit = int(case.vortex is not None and o.wind_drag_limit != 0.0035)
    o.windspeed_averaging_minute, o.wind_multiplier = 1, 1.0
    if case.vortex is not None:
        o.windspeed_averaging_minute = case.vortex.avg_minute
        o.wind_multiplier = case.vortex.wind_mult
        o.has_nws08 = int(case.vortex.avg_minute != 1 or case.vortex.wind_mult != 1.0)
    nbfr, neta = case.sizes["nbfr"], case.sizes["neta"]
    a = case.arrays
    o.nbfr = nbfr
    tabs = {"amig": a["amig"][:nbfr], "ff": a["ff"][:nbfr], "face": a["face"][:nbfr],
            "emo": a["emo"][:nbfr, :neta], "efa": a["efa"][:nbfr, :neta]}
    if case.flux is not None:
        o.nffr = case.flux.famig.size
        tabs.update(famig=case.flux.famig, fff=case.flux.fff, fface=case.flux.fface,
                    qnam=case.flux.qnam, qnph=case.flux.qnph)
        if case.flux.enam is not None:
            tabs.update(enam=case.flux.enam, enph=case.flux.enph)
    return adcirc_io.Fort15(o, [], [f"C{k + 1}" for k in range(nbfr)],
                            [f"F{k + 1}" for k in range(o.nffr)], [], tabs)


# --------------------------------------------------------------------------
# Named cases
# --------------------------------------------------------------------------

M2_PERIOD = 44712.0
K1_PERIOD = 86164.0


def channel_case(dt: float = 5.0, amp: float = 0.5, vortex: bool = False,
                 river: float | None = None, river_type: int = 2, radiation: bool = False,
                 zero_gradient: int = 0, flux_settling: float = 0.0, river_eta: float = 0.05,
                 elev_series: float = 0.0, flux_series: float = 0.0, series_hours: float = 6.0,
                 barrier: float | None = None, barrier_type: int = 3,
                 levee: float | None = None, levee_type: int = 4, pipe=None,
                 prep: MeshPrep | None = None, **kw) -> Case:
    """Tidal channel: 121x41 nodes, 20 m -> 5 m, M2 0.5 m, dt 5 s.  With
    `vortex`, a small Holland vortex (Rmax 8 km) crosses the channel.  With
    `river` [m^2/s per unit width], the closed east end becomes a
    specified-flux boundary (IBTYPE `river_type`, 2 or 22) carrying that
    steady inflow, ramped in over 0.02 days; IBTYPE 52 (river radiation)
    with `flux_settling` > 0 [days] holds the tide until the river flux has
    settled (NRAMP 2); IBTYPE 32 (coupled flux and radiation) also takes
    the steady elevation `river_eta` [m].  With `radiation`, the east end is a radiation
    boundary (IBTYPE 30) the tide leaves through; with `zero_gradient` 40
    (or True) or 41, a zero-normal-velocity-gradient boundary of that type.
    With `elev_series` [s], the open boundary takes no periodic tide (NBFR
    0) but a fort.19 series of that record interval: the M2 sampled at the
    record times with a phase that varies along the boundary, plus a
    set-up of 0.1 m per hour.  With `flux_series` [s] (and `river`), the
    river flux comes from a fort.20 series of that interval (NFFR 0):
    the steady inflow modulated by 50 % with a one-hour period.  Series
    cover `series_hours` of simulated time.  With `barrier` [m above datum],
    the east end is an external barrier (IBTYPE `barrier_type`, 3, 13 or
    23) with that crest height and a discharge coefficient of 1: water
    leaves over it once it stands 6 cm above the crest.  With `levee` [m
    above datum], an internal barrier (IBTYPE `levee_type`, 4 or 24) with
    that crest crosses the channel at x = 30 km and a dry polder at datum
    level lies east of it (meshgen.levee_channel_mesh); for levee_type 5 or
    25, `pipe` = (crown height [m above datum], friction coefficient,
    diameter [m]) gives every pair a pipe under the crest."""
    from .meshgen import channel_mesh, levee_channel_mesh
    raw = channel_mesh() if levee is None else levee_channel_mesh(levee, levee_type, pipe=pipe)
    if river is not None or radiation or zero_gradient or barrier is not None:
        nx, ny = 121, 41
        nid = lambda i, j: i * ny + j
        south = np.array([nid(i, 0) for i in range(nx)])
        east = np.array([nid(nx - 1, j) for j in range(ny)])
        north = np.array([nid(i, ny - 1) for i in range(nx - 1, -1, -1)])
        zg = 40 if zero_gradient is True else int(zero_gradient)
        east_type = 30 if radiation else (zg if zg else river_type)
        if barrier is not None:
            east_type = barrier_type
            raw.barriers = {1: (np.full(east.size, float(barrier)), np.ones(east.size))}
        raw.land_segments = [(0, south), (east_type, east), (0, north)]
    neta = raw.open_nodes.size
    tides = [(2.0 * math.pi / M2_PERIOD, 0.0, 1.0, np.full(neta, amp), np.zeros(neta))]
    if elev_series > 0:
        tides = []
    if vortex:
        kw.setdefault("nws", 8)
    params = default_params(dt, **kw)
    sched = Schedule(dt=dt, dramp=0.5, dramp_mete=0.02 if vortex else 0.5, dramp_extflux=0.02,
                     nramp=2 if flux_settling > 0 else 1, flux_settling_time=flux_settling)
    case = build_case(raw, params, sched, tides, prep=prep)
    if river is not None:
        lbc = case.arrays["lbcodei"]
        nv = lbc.size
        qnam = np.zeros((1, nv))
        qnam[0, (lbc == 2) | (lbc == 12) | (lbc == 22) | (lbc == 32) | (lbc == 52)] = river
        enam = np.where(lbc == 32, river_eta, 0.0)[None, :] if (lbc == 32).any() else None
        case.flux = Flux(np.zeros(1), np.zeros(1), np.ones(1), np.zeros(1), qnam, np.zeros((1, nv)),
                         flux_settling_it=sched.flux_settling_it, enam=enam,
                         enph=None if enam is None else np.zeros((1, nv)))
    if elev_series > 0:
        nrec = int(math.ceil(series_hours * 3600.0 / elev_series)) + 2
        t = np.arange(nrec)[:, None] * elev_series
        phase = np.linspace(0.0, 0.3, neta)[None, :]
        vals = amp * np.cos(2.0 * math.pi / M2_PERIOD * t - phase) + 0.1 * t / 3600.0
        case.elev_series = Series(float(elev_series), vals)
    if flux_series > 0 and case.flux is not None:
        f = case.flux
        nrec = int(math.ceil(series_hours * 3600.0 / flux_series)) + 2
        t = np.arange(nrec)[:, None] * flux_series
        mod = 1.0 + 0.5 * np.sin(2.0 * math.pi * t / 3600.0)
        lbc = case.arrays["lbcodei"]
        on = ((lbc == 2) | (lbc == 12) | (lbc == 22) | (lbc == 32))[None, :]
        q = np.where(on, f.qnam[0][None, :] * mod, 0.0)
        e = None
        if f.enam is not None:
            e = np.where((lbc == 32)[None, :], f.enam[0][None, :] * mod, 0.0)
        case.flux = None
        case.flux_series = Series(float(flux_series), q, e,
                                  flux_settling_it=sched.flux_settling_it)
    if vortex:
        case.vortex = straight_track(30.3e3, 3.7e3, 80.0, 6.0, 960.0, 8.0, 1.3, hours=12.0,
                                     interval_h=3.0)
    return case


def beach_case(dt: float = 2.0, amp: float = 0.5, period: float = 10800.0,
               prep: MeshPrep | None = None, **kw) -> Case:
    """Small beach channel with wetting and drying (parity case).

    A three-hour boundary oscillation starting at mean level on the rise
    floods and drains the upper beach within a few hundred steps.
    """
    from .meshgen import beach_mesh
    raw = beach_mesh()
    neta = raw.open_nodes.size
    tides = [(2.0 * math.pi / period, 0.0, 1.0, np.full(neta, amp), np.zeros(neta))]
    params = default_params(dt, **kw)
    sched = Schedule(dt=dt, statim=0.0, reftim=0.25 * period / 86400.0, nramp=0)
    return build_case(raw, params, sched, tides, prep=prep)


def quarter_annulus_case(dt: float = 100.0, amp: float = 0.3048, tau: float = 1.0e-4,
                         tau0: float = 1.0e-3, nr: int = 21, nth: int = 31,
                         prep: MeshPrep | None = None, **kw) -> Case:
    """Linear tide in the quarter-annular harbour (meshgen.quarter_annulus_mesh):
    M2 of `amp` on the outer arc, linear bottom friction `tau` (NOLIBF = 0),
    no advection, no finite-amplitude terms (H = DP), no Coriolis, no
    lateral viscosity, ramped over half a day.  Its periodic state has the
    closed-form solution of `quarter_annulus_solution`."""
    from .meshgen import quarter_annulus_mesh
    raw = quarter_annulus_mesh(nr, nth)
    neta = raw.open_nodes.size
    tides = [(2.0 * math.pi / M2_PERIOD, 0.0, 1.0, np.full(neta, amp), np.zeros(neta))]
    kw = dict(dict(ifnlfa=0, ifnlct=0, ifnlcat=0, nolifa=0, iflinbf=1, ifnlbf=0, ifhybf=0), **kw)
    params = default_params(dt, **kw)
    sched = Schedule(dt=dt, dramp=0.5, dramp_mete=0.5)
    return build_case(raw, params, sched, tides, cf=tau, tau0=tau0, eslm=0.0, cori=0.0, prep=prep)


def quarter_annulus_solution(r, meta: dict, amp: float = 0.3048, tau: float = 1.0e-4,
                             g: float = G_DEFAULT):
    """Amplitude and phase (eta = A cos(w t - phase)) of the linear periodic
    tide in the quarter annulus, depth h = h1 (r / r1)^2, no flow through
    r = r1 and eta = amp cos(w t) at r = r2 (Lynch and Gray, 1978): with
    eta = Re(E(r) exp(i w t)), the linear equations with bottom friction tau
    give h1/r1^2 (r^2 E'' + 3 r E') = (-w^2 + i w tau) / g E, so E = a r^s1 +
    b r^s2 with s^2 + 2 s - k = 0, k = (-w^2 + i w tau) r1^2 / (g h1)."""
    w = 2.0 * math.pi / M2_PERIOD
    r1, r2, h1 = meta["r1"], meta["r2"], meta["h1"]
    k = (-w * w + 1j * w * tau) * r1 * r1 / (g * h1)
    q = np.sqrt(1.0 + k + 0j)
    s1, s2 = -1.0 + q, -1.0 - q
    # E'(r1) = 0, E(r2) = amp (radii scaled by r1 to keep the powers tame)
    x2 = r2 / r1
    M = np.array([[s1, s2], [x2 ** s1, x2 ** s2]], dtype=complex)
    a, b = np.linalg.solve(M, np.array([0.0, amp], dtype=complex))
    x = np.asarray(r, np.float64) / r1
    E = a * x ** s1 + b * x ** s2
    return np.abs(E), -np.angle(E)


def surge_case(seed: int = 2024, target_nodes: int = 600_000, dt: float = 1.0,
               vortex: bool = True, prep: MeshPrep | None = None, raw=None,
               tau0: float = -1.0, tide_scale: float = 1.0, cf: float = 0.0025,
               eslm: float = 50.0, **kw) -> Case:
    """Graded ~600k-node storm-surge mesh, M2 + K1 on the open boundary and a
    Holland vortex (pc 940 hPa, Rmax 40 km, B 1.3) on a straight northward
    track at 5 m/s that makes landfall on the coast (y ~ 640 km) after
    about 19 h.

    The settings the benchmark specification leaves open are those of an
    ADCIRC surge run over wide tidal flats: hybrid bottom friction (fort.15
    NOLIBF = 2: CF = 0.0025, HBREAK = 2 m, FTHETA = 10, FGAMMA = 1/3,
    nodalattr.F:2399-2413), lateral viscosity ESLM = 50 m^2/s, the wet/dry
    slope limiter SLIM = 1e-4 (wetdry.F:1561-1652) and TAU0 = -1 (0.020 at
    depths of 10 m or less, 0.005 deeper).  With quadratic friction,
    ESLM = 5 and no limiter, the draining flats (currents above 2 m/s in
    0.3 m of water) grow a grid-scale instability within 4 to 6 hours; these
    settings keep the whole day and the landfall surge of 6-8 m stable."""
    params_kw = dict(ifnlbf=0, ifhybf=1, hbreak=2.0, ftheta=10.0, fgamma=1.0 / 3.0, slim=1.0e-4)
    params_kw.update(kw)
    kw = params_kw
    from .meshgen import surge_mesh
    if raw is None:
        raw = surge_mesh(seed=seed, target_nodes=target_nodes)
    neta = raw.open_nodes.size
    xo = raw.x[raw.open_nodes] / raw.meta["lx"]
    tides = [
        (2.0 * math.pi / M2_PERIOD, 0.0, 1.0, tide_scale * (0.5 + 0.1 * xo), np.deg2rad(20.0 * xo)),
        (2.0 * math.pi / K1_PERIOD, 0.0, 1.0, tide_scale * (0.2 + 0.05 * xo), np.deg2rad(10.0 * xo)),
    ]
    if vortex:
        kw.setdefault("nws", 8)
    params = default_params(dt, **kw)
    case = build_case(raw, params, Schedule(dt=dt, dramp=0.25, dramp_mete=0.25), tides, prep=prep,
                      tau0=tau0, cf=cf, eslm=eslm)
    if vortex:
        case.vortex = straight_track(0.5 * raw.meta["lx"] + 1234.5, 300e3 + 678.9, 90.0, 5.0,
                                     940.0, 40.0, 1.3, hours=30.0)
    return case


# --------------------------------------------------------------------------
# Device-resident model
# --------------------------------------------------------------------------

class AdcError(RuntimeError):
    pass


def _check(rc, what):
    if rc != 0:
        raise AdcError(f"{what} failed with status {rc}: {_lib.last_error()}")


class GpuModel:
    """The device-resident step behind the reference's subroutine boundary."""

    def __init__(self, case: Case, prec: int = _lib.ADC_PREC_FP64):
        self.lib = _lib.load()
        self.case = case
        self._p = case.params_struct()
        self._a = case.arrays_struct()
        h = C.c_void_p()
        _check(self.lib.adc_gpu_bind(C.byref(self._p), C.byref(self._a), prec, C.byref(h)),
               "adc_gpu_bind")
        self.h = h
        if case.vortex is not None:
            v, arr = case.vortex.struct()
            _check(self.lib.adc_set_vortex(self.h, C.byref(v)), "adc_set_vortex")
        if case.flux is not None:
            f, keep = case.flux.struct()
            _check(self.lib.adc_set_flux(self.h, C.byref(f)), "adc_set_flux")
        for attr in ("elev_series", "flux_series"):
            ser = getattr(case, attr)
            if ser is not None:
                sv, keep = ser.struct()
                fn = "adc_set_" + attr
                _check(getattr(self.lib, fn)(self.h, C.byref(sv)), fn)

    def close(self):
        if self.h:
            self.lib.adc_gpu_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def hotstart_write(self, path) -> None:
        _check(self.lib.adc_hotstart_write(self.h, str(path).encode()), "adc_hotstart_write")

    def hotstart_read(self, path) -> None:
        _check(self.lib.adc_hotstart_read(self.h, str(path).encode()), "adc_hotstart_read")

    def step(self, it: int) -> AdcStepOut:
        s = self.case.schedule.step(it)
        out = AdcStepOut()
        _check(self.lib.adc_timestep(self.h, C.byref(s), C.byref(out)), "adc_timestep")
        return out

    def run(self, it0: int, n: int):
        steps = self.case.schedule.steps(it0, n)
        numitr = np.zeros(n, np.int32)
        last = AdcStepOut()
        _check(self.lib.adc_run(self.h, n, steps, ptr(numitr, ip_), C.byref(last)), "adc_run")
        return numitr, last

    def sync_to_host(self):
        _check(self.lib.adc_sync_to_host(self.h), "adc_sync_to_host")
        return self.case.state()

    def scalars(self) -> dict:
        """Step-to-step module scalars (adc_get_scalars)."""
        sc = _lib.AdcScalars()
        _check(self.lib.adc_get_scalars(self.h, C.byref(sc)), "adc_get_scalars")
        return {k: getattr(sc, k) for k, _ in sc._fields_ if k != "pad_"}

    def phase_times(self):
        v = [C.c_double() for _ in range(5)]
        self.lib.adc_phase_times(self.h, *[C.byref(t) for t in v])
        return dict(zip(("shift", "gwce", "jcg", "wetdry", "momentum"), [t.value for t in v]))

    # learned initial guess (adc_set_predictor and friends)
    def set_predictor(self, params: np.ndarray) -> None:
        v = np.ascontiguousarray(params, np.float32)
        _check(self.lib.adc_set_predictor(self.h, v.ctypes.data_as(C.POINTER(C.c_float)), v.size),
               "adc_set_predictor")

    def get_predictor(self) -> np.ndarray:
        v = np.zeros(self.lib.adc_predictor_nparams(), np.float32)
        _check(self.lib.adc_get_predictor(self.h, v.ctypes.data_as(C.POINTER(C.c_float)), v.size),
               "adc_get_predictor")
        return v

    def predictor_train(self, on: bool, lr: float = 1e-3) -> None:
        _check(self.lib.adc_predictor_train(self.h, 1 if on else 0, float(lr)), "adc_predictor_train")

    def predictor_stats(self):
        loss = C.c_double(0.0)
        n = C.c_longlong(0)
        _check(self.lib.adc_predictor_stats(self.h, C.byref(loss), C.byref(n)), "adc_predictor_stats")
        return loss.value, n.value

    def predictor_forward(self, hidden: bool = False):
        g = np.zeros(self.case.sizes["np"])
        h = np.zeros(self.case.sizes["np"] * 64, np.float32) if hidden else None
        _check(self.lib.adc_predictor_forward(self.h, ptr(g, dp_),
                                              h.ctypes.data_as(C.POINTER(C.c_float)) if hidden else None),
               "adc_predictor_forward")
        return (g, h.reshape(-1, 64)) if hidden else g

    def predictor_gradient(self) -> np.ndarray:
        v = np.zeros(self.lib.adc_predictor_nparams(), np.float32)
        _check(self.lib.adc_predictor_gradient(self.h, v.ctypes.data_as(C.POINTER(C.c_float)), v.size),
               "adc_predictor_gradient")
        return v

    def predictor_gradient_at(self, target: np.ndarray) -> np.ndarray:
        t = np.ascontiguousarray(target, np.float64)
        v = np.zeros(self.lib.adc_predictor_nparams(), np.float32)
        _check(self.lib.adc_predictor_gradient_at(self.h, ptr(t, dp_),
                                                  v.ctypes.data_as(C.POINTER(C.c_float)), v.size),
               "adc_predictor_gradient_at")
        return v

    def warm_start_stats(self):
        u, f = C.c_longlong(0), C.c_longlong(0)
        _check(self.lib.adc_warm_start_stats(self.h, C.byref(u), C.byref(f)), "adc_warm_start_stats")
        return u.value, f.value

    KERNEL_SPANS = ("lhs_elem", "lhs_gather", "rhs_elem", "rhs_gather", "jcg", "wetdry",
                    "mom_elem", "mom_node")

    def kernel_times(self) -> dict:
        """Device ms of single kernels of the last adc_timestep."""
        v = np.zeros(len(self.KERNEL_SPANS))
        _check(self.lib.adc_kernel_times(self.h, ptr(v, dp_), v.size), "adc_kernel_times")
        return dict(zip(self.KERNEL_SPANS, v.tolist()))

    def launches(self) -> int:
        return int(self.lib.adc_launch_count(self.h))

    def last_run_ms(self) -> float:
        return float(self.lib.adc_last_run_ms(self.h))
