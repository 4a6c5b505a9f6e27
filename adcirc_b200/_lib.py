"""ctypes binding of libadcgpu (include/adcgpu.h)."""
from __future__ import annotations

import ctypes as C
import os
import pathlib

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = _HERE / "lib" / "libadcgpu.so"

dp_ = C.POINTER(C.c_double)
ip_ = C.POINTER(C.c_int)

ADC_OK = 0
ADC_ERR_DIAG = 1
ADC_ERR_ARG = -1
ADC_ERR_MESH = -2
ADC_ERR_CUDA = -3
ADC_ERR_NOMEM = -4
ADC_ERR_TIMEOUT = -5
ADC_ERR_UNSUPPORTED = -6
ADC_PREC_FP64 = 0
ADC_PREC_MIXED = 1
ADC_WARM_START = 2
ADC_LEARNED_START = 32
ADC_F32_ASSEMBLY = 4
ADC_F32_SPMV = 8
ADC_F32_MOMENTUM = 16


class AdcParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "dt", "g", "a00", "b00", "c00", "h0", "velmin", "slim", "hbreak", "ftheta",
        "fgamma", "convcr", "prbckgrnd_mh2o")] + [(n, C.c_int) for n in (
            "ifnlfa", "ifnlct", "ifnlcat", "nolifa", "iflinbf", "ifnlbf", "ifhybf", "itmax",
            "nws", "ifwind", "isldia", "pad_")]


ARRAY_FIELDS = [
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


class AdcArrays(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("np", "ne", "mnei", "neta", "nbfr", "nvel", "nvelme",
                                        "nbou")] + ARRAY_FIELDS


class AdcStep(C.Structure):
    _fields_ = [("it", C.c_int), ("pad_", C.c_int), ("timeloc", C.c_double),
                ("timeh", C.c_double), ("rampelev", C.c_double), ("rampmete", C.c_double),
                ("rampextflux", C.c_double), ("rampintflux", C.c_double)]


class AdcFlux(C.Structure):
    _fields_ = [("nffr", C.c_int), ("flux_settling_it", C.c_int)] + [
        (n, dp_) for n in ("famig", "fper", "fff", "fface", "qnam", "qnph", "enam", "enph")]


class AdcSeries(C.Structure):
    _fields_ = [("nrec", C.c_int), ("flux_settling_it", C.c_int), ("interval", C.c_double),
                ("start_time", C.c_double), ("values", dp_), ("values2", dp_)]


class AdcVortexFix(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("time", "x", "y", "cpress", "vmax", "rmw", "tvx", "tvy")]


class AdcFort22Opts(C.Structure):
    _fields_ = [("irefyr", C.c_int), ("irefmo", C.c_int), ("irefday", C.c_int),
                ("irefhr", C.c_int), ("slam0", C.c_double), ("sfea0", C.c_double),
                ("rnday", C.c_double)]


class AdcFort67(C.Structure):
    _fields_ = [("im", C.c_int), ("it", C.c_int), ("np", C.c_int), ("ne", C.c_int),
                ("timeloc", C.c_double)] + [(n, dp_) for n in ("eta1", "eta2", "etadisc", "uu2",
                                                               "vv2", "ch1")] + [
                ("nodecode", ip_), ("noff", ip_)]


class AdcVortex(C.Structure):
    _fields_ = [("nfix", C.c_int), ("avg_minute", C.c_int), ("hemisphere", C.c_int),
                ("pad_", C.c_int)] + [(n, C.c_double) for n in (
                    "start_time", "bladj", "rho_air", "wind_mult", "drag_limit")] + [
                ("fix", C.POINTER(AdcVortexFix))]


class AdcStepOut(C.Structure):
    _fields_ = [("numitr", C.c_int), ("ier", C.c_int), ("ncchange", C.c_int),
                ("status", C.c_int), ("ep", C.c_double), ("zeta", C.c_double),
                ("cme", C.c_double), ("n_w1_events", C.c_int), ("pad_", C.c_int)]


class AdcScalars(C.Structure):
    _fields_ = [("ncchange", C.c_int), ("q1", C.c_int), ("vortex_counter", C.c_int),
                ("pad_", C.c_int), ("ep", C.c_double), ("rparm1", C.c_double),
                ("rparm2", C.c_double), ("vortex_wtratio", C.c_double)]


class AdcOutputSpec(C.Structure):
    _fields_ = [("nout", C.c_int), ("nspool", C.c_int), ("touts", C.c_double), ("toutf", C.c_double)]


_F15_INTS = ("nfover nabout nscreen ihot ics im nolibf nolifa nolica nolicat nwp ncor ntip nws nramp "
             "nodedrymin nodewetmin storm_number irefyr irefmo irefday irefhr ntif nbfr nffr nfreq "
             "nstae nstav nstac nstam nhainc nhase nhasv nhage nhagv nhstar nhsinc ititer isldia "
             "itmax has_slim has_wind_drag_limit").split()
_F15_REALS = ("bladj g tau0 tau0_min tau0_max dtdp statim reftim rnday dramp dramp_extflux "
              "flux_settling_time dramp_intflux dramp_elev dramp_tip dramp_mete dramp_wrad "
              "dunramp_mete a00 b00 c00 h0 velmin slam0 sfea0 tau cf hbreak ftheta fgamma eslm eslc "
              "cori anginn thas thaf fmv convcr slim wind_drag_limit").split()


class AdcFort15(C.Structure):
    """adc_fort15_t (include/adcgpu.h)."""
    _fields_ = ([("rundes", C.c_char * 88), ("runid", C.c_char * 88)] +
                [(n, C.c_int) for n in _F15_INTS] + [(n, C.c_double) for n in _F15_REALS] +
                [(n, AdcOutputSpec) for n in ("oute", "outv", "outc", "outm", "outge", "outgv",
                                              "outgc", "outgw")] +
                [("has_nws08", C.c_int), ("windspeed_averaging_minute", C.c_int),
                 ("wind_multiplier", C.c_double)])


class AdcFort15Tables(C.Structure):
    """adc_fort15_tables_t (include/adcgpu.h)."""
    _fields_ = ([(n, dp_) for n in ("tpk amigt etrf fft facet amig ff face emo efa famig fff fface "
                                    "qnam qnph enam enph hafreq haff haface xel yel xev yev xem "
                                    "yem").split()] +
                [(n, C.c_char_p) for n in ("tiptag", "bountag", "fbountag", "namefr")])


_lib = None


def load():
    """Load the in-tree libadcgpu.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m adcirc_b200.build` first")
    lib = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    sig = {
        "adc_mesh_geometry": (C.c_int, [C.c_int, C.c_int, dp_, dp_, ip_, dp_, dp_, dp_]),
        "adc_mesh_mnei": (C.c_int, [C.c_int, C.c_int, ip_]),
        "adc_mesh_neighb": (C.c_int, [C.c_int, C.c_int, C.c_int, dp_, dp_, ip_, ip_, ip_, ip_]),
        "adc_mesh_csr_positions": (C.c_int, [C.c_int, C.c_int, C.c_int, ip_, ip_, C.c_int, ip_]),
        "adc_boundary_setup": (C.c_int, [C.c_int, dp_, dp_, C.c_int, ip_, ip_, ip_, C.c_double,
                                          C.c_int, ip_, ip_, ip_, dp_, dp_, ip_, ip_, dp_]),
        "adc_mesh_neitabele": (C.c_int, [C.c_int, C.c_int, C.c_int, ip_, ip_, ip_, ip_]),
        "adc_zng_setup": (C.c_int, [C.c_int, C.c_int, dp_, dp_, ip_, C.c_int, ip_, ip_, dp_, C.c_int, ip_, ip_, dp_, dp_, ip_, dp_, dp_, dp_]),
        "adc_coldstart": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, dp_, ip_, dp_, dp_,
                                     dp_, ip_, ip_, ip_, ip_, dp_]),
        "adc_jcg": (None, [ip_, ip_, ip_, ip_, dp_, dp_, dp_, ip_, ip_, dp_, ip_, dp_, ip_]),
        "adc_dfault": (None, [ip_, dp_]),
        "adc_jcg_reset": (None, []),
        "adc_jcg_noalloc": (None, [ip_, ip_, ip_, ip_, dp_, dp_, dp_, ip_, ip_, dp_, ip_, dp_, ip_]),
        "adc_gpu_bind": (C.c_int, [C.POINTER(AdcParams), C.POINTER(AdcArrays), C.c_int,
                                    C.POINTER(vp)]),
        "adc_gpu_free": (C.c_int, [vp]),
        "adc_shift_friction": (C.c_int, [vp, C.POINTER(AdcStep)]),
        "adc_gwce_new": (C.c_int, [vp, C.POINTER(AdcStep), C.POINTER(AdcStepOut)]),
        "adc_wetdry": (C.c_int, [vp, C.POINTER(AdcStep), C.POINTER(AdcStepOut)]),
        "adc_momentum": (C.c_int, [vp, C.POINTER(AdcStep)]),
        "adc_timestep": (C.c_int, [vp, C.POINTER(AdcStep), C.POINTER(AdcStepOut)]),
        "adc_run": (C.c_int, [vp, C.c_int, C.POINTER(AdcStep), ip_, C.POINTER(AdcStepOut)]),
        "adc_sync_to_host": (C.c_int, [vp]),
        "adc_sync_from_host": (C.c_int, [vp]),
        "adc_set_met": (C.c_int, [vp, dp_, dp_, dp_]),
        "adc_set_vortex": (C.c_int, [vp, C.POINTER(AdcVortex)]),
        "adc_fort67_write": (C.c_int, [C.c_char_p, C.POINTER(AdcFort67)]),
        "adc_fort67_read": (C.c_int, [C.c_char_p, C.POINTER(AdcFort67)]),
        "adc_fort22_read": (C.c_int, [C.c_char_p, C.POINTER(AdcFort22Opts), ip_,
                                      C.POINTER(AdcVortexFix)]),
        "adc_set_flux": (C.c_int, [vp, C.POINTER(AdcFlux)]),
        "adc_set_elev_series": (C.c_int, [vp, C.POINTER(AdcSeries)]),
        "adc_set_flux_series": (C.c_int, [vp, C.POINTER(AdcSeries)]),
        "adc_fort19_read": (C.c_int, [C.c_char_p, C.c_int, ip_, dp_, dp_]),
        "adc_fort20_read": (C.c_int, [C.c_char_p, C.c_int, ip_, ip_, dp_, dp_, dp_]),
        "adc_fort14_dims": (C.c_int, [C.c_char_p, ip_]),
        "adc_fort14_read": (C.c_int, [C.c_char_p, C.c_char_p, dp_, dp_, dp_, ip_, ip_, ip_, ip_, ip_, ip_]),
        "adc_fort15_read": (C.c_int, [C.c_char_p, C.c_int, C.c_int, ip_, C.POINTER(AdcFort15),
                                      C.POINTER(AdcFort15Tables)]),
        "adc_fort15_write": (C.c_int, [C.c_char_p, C.POINTER(AdcFort15), C.c_int, C.c_int, ip_,
                                       C.POINTER(AdcFort15Tables)]),
        "adc_fort14_write": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_int, dp_, dp_, dp_, ip_,
                                       C.c_int, ip_, ip_, C.c_int, ip_, ip_, ip_]),
        "adc_fort14_write_barriers": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_int, dp_, dp_,
                                                dp_, ip_, C.c_int, ip_, ip_, C.c_int, ip_, ip_, ip_,
                                                dp_, dp_, ip_, dp_, dp_, dp_, dp_, dp_, dp_]),
        "adc_fort14_internal_barriers": (C.c_int, [C.c_char_p, ip_, dp_, dp_, dp_, dp_, dp_, dp_]),
        "adc_fort14_barriers": (C.c_int, [C.c_char_p, dp_, dp_]),
        "adc_fort6x_header": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int,
                                        C.c_int, C.c_double, C.c_int, C.c_int]),
        "adc_fort6x_append": (C.c_int, [C.c_char_p, C.c_double, C.c_int, C.c_int, dp_, dp_, ip_,
                                        C.c_double]),
        "adc_selftest_div_const": (C.c_int, [C.c_longlong, C.c_ulonglong, C.POINTER(C.c_longlong)]),
        "adc_hotstart_write": (C.c_int, [vp, C.c_char_p]),
        "adc_hotstart_read": (C.c_int, [vp, C.c_char_p]),
        "adc_warm_start_stats": (C.c_int, [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
        "adc_phase_times": (C.c_int, [vp, dp_, dp_, dp_, dp_, dp_]),
        "adc_launch_count": (C.c_int64, [vp]),
        "adc_get_scalars": (C.c_int, [vp, C.POINTER(AdcScalars)]),
        "adc_kernel_times": (C.c_int, [vp, dp_, C.c_int]),
        "adc_set_jcg_blocks": (C.c_int, [vp, C.c_int]),
        "adc_jcg_layout": (C.c_int, [vp, ip_, ip_]),
        "adc_ensemble_create": (C.c_int, [C.c_int, C.POINTER(vp), C.POINTER(vp)]),
        "adc_ensemble_run": (C.c_int, [vp, C.c_int, C.POINTER(AdcStep), ip_, C.POINTER(AdcStepOut)]),
        "adc_ensemble_last_ms": (C.c_double, [vp]),
        "adc_ensemble_free": (C.c_int, [vp]),
        "adc_predictor_nparams": (C.c_int, []),
        "adc_set_predictor": (C.c_int, [vp, C.POINTER(C.c_float), C.c_int]),
        "adc_get_predictor": (C.c_int, [vp, C.POINTER(C.c_float), C.c_int]),
        "adc_predictor_train": (C.c_int, [vp, C.c_int, C.c_float]),
        "adc_predictor_stats": (C.c_int, [vp, dp_, C.POINTER(C.c_longlong)]),
        "adc_predictor_forward": (C.c_int, [vp, dp_, C.POINTER(C.c_float)]),
        "adc_predictor_gradient": (C.c_int, [vp, C.POINTER(C.c_float), C.c_int]),
        "adc_predictor_gradient_at": (C.c_int, [vp, dp_, C.POINTER(C.c_float), C.c_int]),
        "adc_last_run_ms": (C.c_double, [vp]),
        "adc_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    """Names declared in include/adcgpu.h (used by the ABI test)."""
    import re
    hdr = (_HERE.parent / "include" / "adcgpu.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(adc_\w+)\s*\(", hdr, re.M)))


def ptr(a, typ):
    return a.ctypes.data_as(typ)


def last_error() -> str:
    s = load().adc_last_error()
    return s.decode() if s else ""
