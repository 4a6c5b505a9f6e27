"""ctypes wrapper of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU legs.  It restates the reference Fortran serially in FP64
and is the checker for the CUDA library; the product never calls it.
Parity against the reference binary is unpinned (no Fortran compiler and
no reference golden vectors exist for this path); see oracle.h.
"""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
LIB_MT = HERE / "_build" / "liboracle_mt.so"   # multi-core timing baseline, not the checker

dp_ = C.POINTER(C.c_double)
ip_ = C.POINTER(C.c_int)


class OrcParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "dt", "g", "a00", "b00", "c00", "h0", "velmin", "slim", "hbreak", "ftheta",
        "fgamma", "convcr", "prbckgrnd_mh2o")] + [(n, C.c_int) for n in (
            "ifnlfa", "ifnlct", "ifnlcat", "nolifa", "iflinbf", "ifnlbf", "ifhybf", "itmax",
            "nws", "ifwind", "isldia", "pad_")]


_ARR = [
    ("x", dp_), ("y", dp_), ("dp", dp_), ("nm", ip_), ("nneigh", ip_), ("neitab", ip_),
    ("fdxe", dp_), ("fdye", dp_), ("areas", dp_), ("csr_position", ip_),
    ("tau0var", dp_), ("evm", dp_), ("fric", dp_), ("corif", dp_),
    ("nbd", ip_), ("amig", dp_), ("per", dp_), ("face", dp_), ("ff", dp_),
    ("emo", dp_), ("efa", dp_), ("nbv", ip_), ("lbcodei", ip_), ("csii", dp_), ("siii", dp_),
    ("me2gw", ip_), ("bndlen2o3", dp_),
    ("eta1", dp_), ("eta2", dp_), ("etas", dp_),
    ("uu1", dp_), ("vv1", dp_), ("uu2", dp_), ("vv2", dp_), ("qx1", dp_), ("qy1", dp_),
    ("qx2", dp_), ("qy2", dp_), ("h1", dp_), ("h2", dp_),
    ("tk", dp_), ("tkm", dp_),
    ("nodecode", ip_), ("nnodecode", ip_), ("noff", ip_), ("mju", ip_),
    ("totalarea", dp_), ("alphal", dp_),
    ("wsx1", dp_), ("wsy1", dp_), ("wsx2", dp_), ("wsy2", dp_), ("pr1", dp_), ("pr2", dp_),
    ("coef", dp_), ("obccoef", dp_),
    ("gwce_lv", dp_), ("mom_lv_x", dp_), ("mom_lv_y", dp_),
    ("nelezng", ip_), ("zngif1", dp_), ("zngif2", dp_), ("zngif3", dp_), ("neitabele", ip_),
    ("barlanht", dp_), ("barlancfsp", dp_),
    ("ibconn", ip_), ("barinht", dp_), ("barincfsb", dp_), ("barincfsp", dp_), ("nvell", ip_),
    ("pipeht", dp_), ("pipecoef", dp_), ("pipediam", dp_),
]


class OrcArrays(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("np", "ne", "mnei", "neta", "nbfr", "nvel", "nvelme",
                                        "nbou")] + _ARR


class OrcStep(C.Structure):
    _fields_ = [("it", C.c_int), ("pad_", C.c_int), ("timeloc", C.c_double),
                ("timeh", C.c_double), ("rampelev", C.c_double), ("rampmete", C.c_double),
                ("rampextflux", C.c_double), ("rampintflux", C.c_double)]


class OrcFlux(C.Structure):
    _fields_ = [("nffr", C.c_int), ("flux_settling_it", C.c_int)] + [
        (n, dp_) for n in ("famig", "fper", "fff", "fface", "qnam", "qnph", "enam", "enph")]


class OrcSeries(C.Structure):
    _fields_ = [("nrec", C.c_int), ("flux_settling_it", C.c_int), ("interval", C.c_double),
                ("start_time", C.c_double), ("values", dp_), ("values2", dp_)]


class OrcStepOut(C.Structure):
    _fields_ = [("numitr", C.c_int), ("ier", C.c_int), ("ncchange", C.c_int),
                ("status", C.c_int), ("ep", C.c_double), ("zeta", C.c_double),
                ("cme", C.c_double), ("n_w1_events", C.c_int), ("pad_", C.c_int)]


class OrcVortexFix(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("time", "x", "y", "cpress", "vmax", "rmw", "tvx", "tvy")]


class OrcVortex(C.Structure):
    _fields_ = [("nfix", C.c_int), ("avg_minute", C.c_int), ("hemisphere", C.c_int),
                ("pad_", C.c_int)] + [(n, C.c_double) for n in (
                    "start_time", "bladj", "rho_air", "wind_mult", "drag_limit")] + [
                ("fix", C.POINTER(OrcVortexFix))]


_lib = None
_lib_mt = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load(omp: bool = False):
    """The checker (serial) or, with `omp`, the multi-threaded build (its
    loops split over all host cores) used only as the multi-core CPU
    baseline."""
    global _lib, _lib_mt
    if omp and _lib_mt is not None:
        return _lib_mt
    if not omp and _lib is not None:
        return _lib
    if not (LIB_MT if omp else LIB).exists():
        build()
    lib = C.CDLL(str(LIB_MT if omp else LIB))
    lib.orc_jcg.argtypes = [ip_, ip_, ip_, ip_, dp_, dp_, dp_, ip_, ip_, dp_, ip_, dp_, ip_]
    lib.orc_jcg.restype = None
    lib.orc_dfault.argtypes = [ip_, dp_]
    lib.orc_itpack_reset.argtypes = []
    lib.orc_model_create.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcArrays)]
    lib.orc_model_create.restype = C.c_void_p
    lib.orc_model_destroy.argtypes = [C.c_void_p]
    for f in ("orc_model_step", "orc_model_gwce", "orc_model_wetdry"):
        getattr(lib, f).argtypes = [C.c_void_p, C.POINTER(OrcStep), C.POINTER(OrcStepOut)]
        getattr(lib, f).restype = C.c_int
    for f in ("orc_model_shift_friction", "orc_model_momentum"):
        getattr(lib, f).argtypes = [C.c_void_p, C.POINTER(OrcStep)]
        getattr(lib, f).restype = C.c_int
    lib.orc_model_set_flux.argtypes = [C.c_void_p, C.POINTER(OrcFlux)]
    lib.orc_model_set_flux.restype = C.c_int
    for f in ("orc_model_set_elev_series", "orc_model_set_flux_series"):
        getattr(lib, f).argtypes = [C.c_void_p, C.POINTER(OrcSeries)]
        getattr(lib, f).restype = C.c_int
    lib.orc_model_set_vortex.argtypes = [C.c_void_p, C.POINTER(OrcVortex)]
    lib.orc_model_set_vortex.restype = C.c_int
    lib.orc_model_met.argtypes = [C.c_void_p, C.POINTER(OrcStep)]
    lib.orc_model_met.restype = C.c_int
    lib.orc_model_set_ncchange.argtypes = [C.c_void_p, C.c_int]
    lib.orc_model_get_ncchange.argtypes = [C.c_void_p]
    lib.orc_model_get_ncchange.restype = C.c_int
    lib.orc_model_get_zeta.argtypes = [C.c_void_p]
    lib.orc_model_get_zeta.restype = C.c_double
    lib.orc_coldstart.argtypes = [C.POINTER(OrcParams), C.POINTER(OrcArrays)]
    lib.orc_model_set_scalars.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double,
                                          C.c_double, C.c_int, C.c_int, C.c_double]
    lib.orc_model_set_scalars.restype = None
    sig = {
        "orc_mesh_geometry": [C.c_int, C.c_int, dp_, dp_, ip_, dp_, dp_, dp_],
        "orc_mesh_mnei": [C.c_int, C.c_int, ip_],
        "orc_mesh_neighb": [C.c_int, C.c_int, C.c_int, dp_, dp_, ip_, ip_, ip_, ip_],
        "orc_mesh_csr_positions": [C.c_int, C.c_int, C.c_int, ip_, ip_, C.c_int, ip_],
        "orc_boundary_setup": [C.c_int, dp_, dp_, C.c_int, ip_, ip_, ip_, C.c_double, C.c_int,
                               ip_, ip_, ip_, dp_, dp_, ip_, ip_, dp_],
        "orc_mesh_neitabele": [C.c_int, C.c_int, C.c_int, ip_, ip_, ip_, ip_],
        "orc_zng_setup": [C.c_int, C.c_int, dp_, dp_, ip_, C.c_int, ip_, ip_, dp_, C.c_int, ip_, ip_, dp_, dp_, ip_, dp_, dp_, dp_],
        "orc_coldstart_arrays": [C.c_int, C.c_int, C.c_int, C.c_double, dp_, ip_, dp_, dp_, dp_,
                                 ip_, ip_, ip_, ip_, dp_],
    }
    for name, args in sig.items():
        getattr(lib, name).argtypes = args
        getattr(lib, name).restype = C.c_int
    if omp:
        _lib_mt = lib
    else:
        _lib = lib
    return lib


def _ptr(a, typ):
    return a.ctypes.data_as(typ)


class OracleModel:
    """Serial FP64 oracle stepping a case's arrays in place (its own copy)."""

    def __init__(self, case, omp: bool = False):
        self.lib = load(omp)
        self.case = case
        self.p = OrcParams()
        for k, v in case.params.items():
            setattr(self.p, k, v)
        self.a = OrcArrays()
        for k in ("np", "ne", "mnei", "neta", "nbfr", "nvel", "nvelme", "nbou"):
            setattr(self.a, k, int(case.sizes[k]))
        for name, typ in _ARR:
            arr = case.arrays[name]
            assert arr.flags.f_contiguous
            setattr(self.a, name, _ptr(arr, typ))
        self.h = self.lib.orc_model_create(C.byref(self.p), C.byref(self.a))
        vortex = getattr(case, "vortex", None)
        if vortex is not None:
            self.set_vortex(vortex)
        flux = getattr(case, "flux", None)
        if flux is not None:
            f, keep = flux.struct(OrcFlux)
            if self.lib.orc_model_set_flux(self.h, C.byref(f)) != 0:
                raise ValueError("invalid flux forcing")
        for attr, fn in (("elev_series", "orc_model_set_elev_series"),
                         ("flux_series", "orc_model_set_flux_series")):
            ser = getattr(case, attr, None)
            if ser is not None:
                sv, self._series_keep = ser.struct(OrcSeries)
                if getattr(self.lib, fn)(self.h, C.byref(sv)) != 0:
                    raise ValueError(f"invalid {attr}")

    def set_vortex(self, vortex):
        """vortex: an object with the adcirc_b200.model.Vortex fields."""
        fx = np.ascontiguousarray(vortex.fixes, dtype=np.float64)
        arr = (OrcVortexFix * len(fx))()
        for k, row in enumerate(fx):
            arr[k] = OrcVortexFix(*[float(v) for v in row])
        v = OrcVortex()
        v.nfix, v.avg_minute, v.hemisphere = len(fx), vortex.avg_minute, vortex.hemisphere
        v.start_time, v.bladj, v.rho_air = vortex.start_time, vortex.bladj, vortex.rho_air
        v.wind_mult, v.drag_limit = vortex.wind_mult, vortex.drag_limit
        v.fix = C.cast(arr, C.POINTER(OrcVortexFix))
        rc = self.lib.orc_model_set_vortex(self.h, C.byref(v))
        if rc != 0:
            raise ValueError("invalid vortex track")

    def set_scalars(self, sc: dict):
        """Continue from another implementation's state: `sc` holds the
        fields of adc_scalars_t (the arrays are the case's, set beforehand)."""
        self.lib.orc_model_set_scalars(self.h, int(sc["ncchange"]), float(sc["ep"]),
                                       float(sc["rparm1"]), float(sc["rparm2"]), int(sc["q1"]),
                                       int(sc["vortex_counter"]), float(sc["vortex_wtratio"]))

    def met(self, it):
        """The met phase alone for step `it`; nonzero once past the track."""
        return self.lib.orc_model_met(self.h, C.byref(self._st(it)))

    def close(self):
        if self.h:
            self.lib.orc_model_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _st(self, it):
        s = self.case.schedule.step(it)
        o = OrcStep()
        o.it, o.timeloc, o.timeh, o.rampelev, o.rampmete = s.it, s.timeloc, s.timeh, s.rampelev, s.rampmete
        o.rampextflux, o.rampintflux = s.rampextflux, s.rampintflux
        return o

    def step(self, it) -> OrcStepOut:
        out = OrcStepOut()
        rc = self.lib.orc_model_step(self.h, C.byref(self._st(it)), C.byref(out))
        if rc != 0:
            raise RuntimeError(f"oracle step {it} failed: status {rc}")
        return out

    def run(self, it0, n):
        its = []
        for k in range(n):
            its.append(self.step(it0 + k).numitr)
        return np.asarray(its)

    def shift_friction(self, it):
        self.lib.orc_model_shift_friction(self.h, C.byref(self._st(it)))

    def gwce(self, it) -> OrcStepOut:
        out = OrcStepOut()
        self.lib.orc_model_gwce(self.h, C.byref(self._st(it)), C.byref(out))
        return out

    def wetdry(self, it) -> OrcStepOut:
        out = OrcStepOut()
        self.lib.orc_model_wetdry(self.h, C.byref(self._st(it)), C.byref(out))
        a = self.case.arrays
        a["h2"][:] = a["dp"] + self.case.params["ifnlfa"] * a["eta2"]
        return out

    def momentum(self, it):
        self.lib.orc_model_momentum(self.h, C.byref(self._st(it)))


def jcg(n, ndim, maxnz, jcoef, coef, rhs, u, iparm, rparm):
    """Call the oracle's ITPACK jcg on Fortran-layout arrays (in place)."""
    lib = load()
    nw = 4 * n + 4 * int(iparm[0])
    wksp = np.zeros(nw + 16)
    iwksp = np.zeros(3 * n, np.int32)
    ier = C.c_int(0)
    lib.orc_jcg(C.byref(C.c_int(n)), C.byref(C.c_int(ndim)), C.byref(C.c_int(maxnz)),
                _ptr(jcoef, ip_), _ptr(coef, dp_), _ptr(rhs, dp_), _ptr(u, dp_),
                _ptr(iwksp, ip_), C.byref(C.c_int(nw)), _ptr(wksp, dp_), _ptr(iparm, ip_),
                _ptr(rparm, dp_), C.byref(ier))
    return ier.value


def mesh_prep():
    """The oracle's own table builders (oracle_mesh.cpp), with the argument
    lists of the library's: pass as `prep=` to adcirc_b200.model.build_case
    (or a named case) to build a case without the library."""
    import types
    lib = load()
    return types.SimpleNamespace(
        geometry=lib.orc_mesh_geometry, mnei=lib.orc_mesh_mnei, neighb=lib.orc_mesh_neighb,
        csr_positions=lib.orc_mesh_csr_positions, boundary_setup=lib.orc_boundary_setup,
        coldstart=lib.orc_coldstart_arrays, zng_setup=lib.orc_zng_setup,
        neitabele=lib.orc_mesh_neitabele)


def dfault():
    iparm = np.zeros(12, np.int32)
    rparm = np.zeros(12)
    load().orc_dfault(_ptr(iparm, ip_), _ptr(rparm, dp_))
    return iparm, rparm
