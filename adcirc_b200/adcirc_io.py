"""ADCIRC text files at the edges of the hot path, through libadcgpu's host
functions: fort.14 meshes (read14, mesh.F:319-581), fort.15 model
parameters (READ_INPUT, read_input.F:949-4566) and the full-domain ASCII
outputs fort.63/fort.64 (globalio.F:544-643, 802-930, 1005-1085)."""
from __future__ import annotations

import ctypes as C
import dataclasses
import os

import numpy as np

from . import _lib
from ._lib import dp_, ip_, ptr
from .meshgen import RawMesh

DRY_VALUE = -99999.0   # the reference's alternate value for dry nodes


def _check(rc, what):
    if rc != 0:
        raise OSError(f"{what} failed with status {rc}: {_lib.last_error()}")


def read_fort14(path) -> RawMesh:
    """A fort.14 mesh as a RawMesh (0-based node ids; the elevation
    boundary segments concatenated as NBD; flux segments with IBTYPE)."""
    lib = _lib.load()
    p = os.fsencode(path)
    dims = np.zeros(6, np.int32)
    _check(lib.adc_fort14_dims(p, ptr(dims, ip_)), "adc_fort14_dims")
    npn, ne, nope, neta, nbou, nvel = (int(v) for v in dims)
    x, y, dp = (np.zeros(npn) for _ in range(3))
    nm = np.zeros((ne, 3), np.int32, order="F")
    nvdll = np.zeros(max(nope, 1), np.int32)
    nbdv = np.zeros(max(neta, 1), np.int32)
    nvell = np.zeros(max(nbou, 1), np.int32)
    ibtype = np.zeros(max(nbou, 1), np.int32)
    nbvv = np.zeros(max(nvel, 1), np.int32)
    title = C.create_string_buffer(81)
    _check(lib.adc_fort14_read(p, title, ptr(x, dp_), ptr(y, dp_), ptr(dp, dp_), ptr(nm, ip_),
                               ptr(nvdll, ip_), ptr(nbdv, ip_), ptr(nvell, ip_), ptr(ibtype, ip_),
                               ptr(nbvv, ip_)), "adc_fort14_read")
    bht, bcf = np.zeros(max(nvel, 1)), np.zeros(max(nvel, 1))
    if any(int(t) in (3, 13, 23) for t in ibtype[:nbou]):
        _check(lib.adc_fort14_barriers(p, ptr(bht, dp_), ptr(bcf, dp_)), "adc_fort14_barriers")
    ibc = np.zeros(max(nvel, 1), np.int32)
    iht, icb, icp, pht, pcf, pdm = (np.zeros(max(nvel, 1)) for _ in range(6))
    if any(int(t) in (4, 24, 5, 25) for t in ibtype[:nbou]):
        _check(lib.adc_fort14_internal_barriers(p, ptr(ibc, ip_), ptr(iht, dp_), ptr(icb, dp_),
                                                ptr(icp, dp_), ptr(pht, dp_), ptr(pcf, dp_),
                                                ptr(pdm, dp_)), "adc_fort14_internal_barriers")
    segs, barriers, q = [], {}, 0
    for k in range(nbou):
        n = int(nvell[k])
        segs.append((int(ibtype[k]), nbvv[q:q + n].astype(np.int64) - 1))
        if int(ibtype[k]) in (3, 13, 23):
            barriers[k] = (bht[q:q + n].copy(), bcf[q:q + n].copy())
        if int(ibtype[k]) in (4, 24, 5, 25):
            barriers[k] = (iht[q:q + n].copy(), icb[q:q + n].copy(), icp[q:q + n].copy(),
                           ibc[q:q + n].astype(np.int64) - 1)
        if int(ibtype[k]) in (5, 25):
            barriers[k] += (pht[q:q + n].copy(), pcf[q:q + n].copy(), pdm[q:q + n].copy())
        q += n
    name = title.value.decode(errors="replace").strip() or os.path.basename(os.fsdecode(path))
    meta = {"lx": float(x.max() - x.min()), "ly": float(y.max() - y.min()),
            "open_segments": [int(v) for v in nvdll[:nope]], "source": os.fsdecode(path)}
    return RawMesh(name, x, y, dp, np.asarray(nm, np.int64) - 1,
                   nbdv[:neta].astype(np.int64) - 1, segs, meta, barriers)


def write_fort14(raw: RawMesh, path, title: str | None = None) -> None:
    """Writes a RawMesh as fort.14 (one elevation boundary segment unless
    raw.meta['open_segments'] splits NBD)."""
    lib = _lib.load()
    x, y, dp = (np.ascontiguousarray(a, np.float64) for a in (raw.x, raw.y, raw.dp))
    nm = np.asfortranarray(np.asarray(raw.nm, np.int32) + 1)
    nbdv = np.ascontiguousarray(np.asarray(raw.open_nodes, np.int32) + 1)
    lens = raw.meta.get("open_segments") or ([int(nbdv.size)] if nbdv.size else [])
    nvdll = np.asarray(lens if lens else [0], np.int32)
    ibtype = np.asarray([t for t, _ in raw.land_segments] or [0], np.int32)
    nvell = np.asarray([len(s) for _, s in raw.land_segments] or [0], np.int32)
    nbvv = (np.concatenate([np.asarray(s, np.int32) + 1 for _, s in raw.land_segments])
            if raw.land_segments else np.zeros(1, np.int32))
    nbvv = np.ascontiguousarray(nbvv, np.int32)
    bht, bcf = np.zeros(max(nbvv.size, 1)), np.zeros(max(nbvv.size, 1))
    ibc = np.zeros(max(nbvv.size, 1), np.int32)
    iht, icb, icp, pht, pcf, pdm = (np.zeros(max(nbvv.size, 1)) for _ in range(6))
    q = 0
    for k, (t, nodes) in enumerate(raw.land_segments):
        n = len(nodes)
        if t in (3, 13, 23):
            bht[q:q + n], bcf[q:q + n] = raw.barriers[k]
        if t in (4, 24, 5, 25):
            iht[q:q + n], icb[q:q + n], icp[q:q + n], across = raw.barriers[k][:4]
            ibc[q:q + n] = np.asarray(across) + 1
        if t in (5, 25):
            pht[q:q + n], pcf[q:q + n], pdm[q:q + n] = raw.barriers[k][4:7]
        q += n
    _check(lib.adc_fort14_write_barriers(os.fsencode(path), (title or raw.name).encode()[:80],
                                         int(x.size), int(nm.shape[0]), ptr(x, dp_), ptr(y, dp_),
                                         ptr(dp, dp_), ptr(nm, ip_), len(lens), ptr(nvdll, ip_),
                                         ptr(nbdv, ip_), len(raw.land_segments), ptr(nvell, ip_),
                                         ptr(ibtype, ip_), ptr(nbvv, ip_), ptr(bht, dp_),
                                         ptr(bcf, dp_), ptr(ibc, ip_), ptr(iht, dp_),
                                         ptr(icb, dp_), ptr(icp, dp_), ptr(pht, dp_), ptr(pcf, dp_),
                                         ptr(pdm, dp_)), "adc_fort14_write_barriers")


class Fort6x:
    """fort.63 (irtype 1: elevation) or fort.64 (irtype 2: velocity)."""

    def __init__(self, path, np_: int, irtype: int, dt_out: float, nspool: int, ndsets: int,
                 rundes: str = "adcirc_b200", runid: str = "run", agrid: str = "grid"):
        self.lib = _lib.load()
        self.path = os.fsencode(path)
        self.np, self.irtype = int(np_), int(irtype)
        _check(self.lib.adc_fort6x_header(self.path, rundes.encode(), runid.encode(),
                                          agrid.encode(), int(ndsets), self.np, float(dt_out),
                                          int(nspool), self.irtype), "adc_fort6x_header")

    def append(self, timeloc: float, it: int, v1, v2=None, nodecode=None,
               alternate: float = DRY_VALUE) -> None:
        a = np.ascontiguousarray(v1, np.float64)
        b = None if v2 is None else np.ascontiguousarray(v2, np.float64)
        nc = None if nodecode is None else np.ascontiguousarray(nodecode, np.int32)
        _check(self.lib.adc_fort6x_append(self.path, float(timeloc), int(it), self.np, ptr(a, dp_),
                                          ptr(b, dp_) if b is not None else None,
                                          ptr(nc, ip_) if nc is not None else None,
                                          float(alternate)), "adc_fort6x_append")


# ---------------------------------------------------------------- fort.15
_F15_TABLE_COUNTS = {
    "ntif": ("tpk", "amigt", "etrf", "fft", "facet"),
    "nbfr": ("amig", "ff", "face"),
    "nffr": ("famig", "fff", "fface"),
    "nfreq": ("hafreq", "haff", "haface"),
}
_F15_TAGS = {"ntif": "tiptag", "nbfr": "bountag", "nffr": "fbountag", "nfreq": "namefr"}


@dataclasses.dataclass
class Fort15:
    """A fort.15 file's values: `p` holds every scalar record (an
    adc_fort15_t), the other fields the tables, angles in radians where
    read_input converts them (FACE, EFA, FFACE, QNPH, ENPH, FACET)."""
    p: object
    tiptag: list
    bountag: list
    fbountag: list
    namefr: list
    tables: dict      # name -> array: (NTIF,), (NBFR,), EMO/EFA (NBFR, NETA), QNAM... (NFFR, NVEL)

    def __getattr__(self, name):
        if name in ("p", "tables"):
            raise AttributeError(name)
        if name in self.tables:
            return self.tables[name]
        return getattr(self.p, name)


def _f15_tables(counts: dict, neta: int, nvel: int):
    """Zeroed tables for the given counts and the ctypes struct over them."""
    tabs = {}
    for cnt, names in _F15_TABLE_COUNTS.items():
        for nm in names:
            tabs[nm] = np.zeros(max(counts[cnt], 1))
    nb, nf = max(counts["nbfr"], 1), max(counts["nffr"], 1)
    for nm in ("emo", "efa"):
        tabs[nm] = np.zeros((nb, max(neta, 1)), order="F")
    for nm in ("qnam", "qnph", "enam", "enph"):
        tabs[nm] = np.zeros((nf, max(nvel, 1)), order="F")
    for nm, cnt in (("xel", "nstae"), ("yel", "nstae"), ("xev", "nstav"), ("yev", "nstav"),
                    ("xem", "nstam"), ("yem", "nstam")):
        tabs[nm] = np.zeros(max(counts[cnt], 1))
    tags = {cnt: C.create_string_buffer(16 * max(counts[cnt], 1)) for cnt in _F15_TAGS}
    t = _lib.AdcFort15Tables()
    for nm, a in tabs.items():
        setattr(t, nm, ptr(a, dp_))
    for cnt, field in _F15_TAGS.items():
        setattr(t, field, C.cast(tags[cnt], C.c_char_p))
    return tabs, tags, t


def read_fort15(path, neta: int, lbcodei) -> Fort15:
    """Reads a fort.15 (adc_fort15_read).  neta: NETA of the mesh;
    lbcodei: LBCODEI of the flux-boundary nodes in the reference's order
    (a Case's arrays['lbcodei']), which places the flux records."""
    lib = _lib.load()
    p = os.fsencode(path)
    lbc = np.ascontiguousarray(np.asarray(lbcodei, np.int32).ravel())
    nvel = int(lbc.size)
    o = _lib.AdcFort15()
    _check(lib.adc_fort15_read(p, int(neta), nvel, ptr(lbc, ip_), C.byref(o), None), "adc_fort15_read")
    counts = {k: int(getattr(o, k)) for k in ("ntif", "nbfr", "nffr", "nfreq", "nstae", "nstav", "nstam")}
    tabs, tags, t = _f15_tables(counts, neta, nvel)
    o = _lib.AdcFort15()
    _check(lib.adc_fort15_read(p, int(neta), nvel, ptr(lbc, ip_), C.byref(o), C.byref(t)),
           "adc_fort15_read")

    def taglist(cnt):
        raw = tags[cnt].raw
        return [raw[16 * k:16 * k + 16].split(b"\0", 1)[0].decode(errors="replace")
                for k in range(counts[cnt])]
    for cnt, names in _F15_TABLE_COUNTS.items():
        for nm in names:
            tabs[nm] = tabs[nm][:counts[cnt]]
    tabs["emo"], tabs["efa"] = (tabs[k][:counts["nbfr"], :neta] for k in ("emo", "efa"))
    for k in ("qnam", "qnph", "enam", "enph"):
        tabs[k] = tabs[k][:counts["nffr"], :nvel]
    for k, cnt in (("xel", "nstae"), ("yel", "nstae"), ("xev", "nstav"), ("yev", "nstav"),
                   ("xem", "nstam"), ("yem", "nstam")):
        tabs[k] = tabs[k][:counts[cnt]]
    return Fort15(o, taglist("ntif"), taglist("nbfr"), taglist("nffr"), taglist("nfreq"), tabs)


def write_fort15(path, f: Fort15, neta: int, lbcodei) -> None:
    """Writes `f` as a fort.15 (adc_fort15_write): read_fort15 of the file
    gives back the same values."""
    lib = _lib.load()
    lbc = np.ascontiguousarray(np.asarray(lbcodei, np.int32).ravel())
    nvel = int(lbc.size)
    counts = {k: int(getattr(f.p, k)) for k in ("ntif", "nbfr", "nffr", "nfreq", "nstae", "nstav",
                                                   "nstam")}
    tabs, tags, t = _f15_tables(counts, neta, nvel)
    for nm, a in f.tables.items():
        a = np.asarray(a, np.float64)
        if a.size:
            tabs[nm][tuple(slice(0, s) for s in a.shape)] = a
    for cnt, field in _F15_TAGS.items():
        names = {"ntif": f.tiptag, "nbfr": f.bountag, "nffr": f.fbountag, "nfreq": f.namefr}[cnt]
        buf = b"".join(n.encode()[:15].ljust(16, b"\0") for n in names)
        C.memmove(tags[cnt], buf, min(len(buf), C.sizeof(tags[cnt])))
    _check(lib.adc_fort15_write(os.fsencode(path), C.byref(f.p), int(neta), nvel, ptr(lbc, ip_),
                                C.byref(t)), "adc_fort15_write")


def read_fort19(path, neta: int, start_time: float = 0.0):
    """Reads a fort.19 non-periodic elevation boundary file
    (adc_fort19_read) into a model.Series of (nrec, NETA) records."""
    from .model import Series
    lib = _lib.load()
    p = os.fsencode(path)
    n, inc = C.c_int(0), C.c_double(0.0)
    _check(lib.adc_fort19_read(p, int(neta), C.byref(n), C.byref(inc), None), "adc_fort19_read")
    vals = np.zeros((n.value, int(neta)))
    _check(lib.adc_fort19_read(p, int(neta), C.byref(n), C.byref(inc), ptr(vals, dp_)),
           "adc_fort19_read")
    return Series(inc.value, vals, start_time=start_time)


def read_fort20(path, lbcodei, start_time: float = 0.0, flux_settling_it: int = 0):
    """Reads a fort.20 non-periodic normal-flux file (adc_fort20_read) into a
    model.Series of (nrec, NVEL) fluxes, with the elevations of code-32
    entries as values2 when there are any.  lbcodei: LBCODEI of the
    flux-boundary nodes (a Case's arrays['lbcodei'])."""
    from .model import Series
    lib = _lib.load()
    p = os.fsencode(path)
    lbc = np.ascontiguousarray(np.asarray(lbcodei, np.int32).ravel())
    nv = int(lbc.size)
    n, inc = C.c_int(0), C.c_double(0.0)
    _check(lib.adc_fort20_read(p, nv, ptr(lbc, ip_), C.byref(n), C.byref(inc), None, None),
           "adc_fort20_read")
    q = np.zeros((n.value, nv))
    e = np.zeros((n.value, nv))
    _check(lib.adc_fort20_read(p, nv, ptr(lbc, ip_), C.byref(n), C.byref(inc), ptr(q, dp_),
                               ptr(e, dp_)), "adc_fort20_read")
    return Series(inc.value, q, e if (lbc == 32).any() else None, start_time=start_time,
                  flux_settling_it=flux_settling_it)


def write_fort19(path, series) -> None:
    """Writes a model.Series as a fort.19: the interval, then one value per
    line, record after record (17 significant digits)."""
    with open(path, "w") as f:
        f.write(f"{series.interval!r}\n")
        for rec in np.asarray(series.values):
            f.writelines(f"{float(v)!r}\n" for v in rec)


def write_fort20(path, series, lbcodei) -> None:
    """Writes a model.Series as a fort.20: the interval, then per record one
    line per entry of code 2/12/22 (its flux) or 32 (flux and elevation)."""
    lbc = np.asarray(lbcodei).ravel()
    e = series.values2
    with open(path, "w") as f:
        f.write(f"{series.interval!r}\n")
        for k, rec in enumerate(np.asarray(series.values)):
            for j, lb in enumerate(lbc):
                if lb in (2, 12, 22):
                    f.write(f"{float(rec[j])!r}\n")
                elif lb == 32:
                    ev = 0.0 if e is None else float(e[k, j])
                    f.write(f"{float(rec[j])!r} {ev!r}\n")


def read_fort22(path, irefyr: int, irefmo: int, irefday: int, irefhr: int, slam0: float = 0.0,
                sfea0: float = 0.0, rnday: float = 0.0, **vortex_kw):
    """Reads an NWS = 8 fort.22 (ATCF best-track lines; adc_fort22_read) into
    a model.Vortex: times since the wind reference time IREFYR/IREFMO/
    IREFDAY/IREFHR, centres projected about (SLAM0, SFEA0) [degrees] into mesh
    metres.  `rnday` > 0 requires the track to reach RNDAY days.  vortex_kw
    (bladj, start_time, ...) go to the Vortex."""
    from .model import Vortex
    lib = _lib.load()
    p = os.fsencode(path)
    o = _lib.AdcFort22Opts(int(irefyr), int(irefmo), int(irefday), int(irefhr), float(slam0),
                           float(sfea0), float(rnday))
    n = C.c_int(0)
    _check(lib.adc_fort22_read(p, C.byref(o), C.byref(n), None), "adc_fort22_read")
    arr = (_lib.AdcVortexFix * n.value)()
    _check(lib.adc_fort22_read(p, C.byref(o), C.byref(n), arr), "adc_fort22_read")
    rows = np.array([[getattr(arr[k], f) for f, _ in _lib.AdcVortexFix._fields_]
                     for k in range(n.value)])
    vortex_kw.setdefault("hemisphere", -1 if rows[0, 2] < 0.0 else 1)   # sign(1, lat)
    return Vortex(rows, **vortex_kw)


def write_fort67(path, case, it: int, timeloc: float, im: int = 0, etadisc=None) -> None:
    """Writes a case's state (as adc_sync_to_host leaves it) as the
    reference's binary hotstart file (adc_fort67_write), for a reference run
    to continue from."""
    lib = _lib.load()
    a = case.arrays
    npn, ne = case.sizes["np"], case.sizes["ne"]
    keep = {k: np.ascontiguousarray(a[k], np.float64) for k in ("eta1", "eta2", "uu2", "vv2")}
    nc = np.ascontiguousarray(a["nodecode"], np.int32)
    noff = np.ascontiguousarray(a["noff"], np.int32)
    ed = np.ascontiguousarray(np.zeros(npn) if etadisc is None else etadisc, np.float64)
    h = _lib.AdcFort67(int(im), int(it), npn, ne, float(timeloc), keep["eta1"].ctypes.data_as(dp_),
                       keep["eta2"].ctypes.data_as(dp_), ed.ctypes.data_as(dp_),
                       keep["uu2"].ctypes.data_as(dp_), keep["vv2"].ctypes.data_as(dp_), None,
                       nc.ctypes.data_as(ip_), noff.ctypes.data_as(ip_))
    _check(lib.adc_fort67_write(os.fsencode(path), C.byref(h)), "adc_fort67_write")


def read_fort67(path) -> dict:
    """Reads the reference's binary hotstart file (adc_fort67_read): a dict
    of im, it, timeloc and the arrays eta1, eta2, etadisc, uu2, vv2,
    nodecode, noff (ch1 when IM = 10)."""
    lib = _lib.load()
    p = os.fsencode(path)
    h = _lib.AdcFort67()
    _check(lib.adc_fort67_read(p, C.byref(h)), "adc_fort67_read")
    npn, ne = h.np, h.ne
    out = {k: np.zeros(npn) for k in ("eta1", "eta2", "etadisc", "uu2", "vv2", "ch1")}
    out["nodecode"] = np.zeros(npn, np.int32)
    out["noff"] = np.zeros(ne, np.int32)
    for k in ("eta1", "eta2", "etadisc", "uu2", "vv2", "ch1"):
        setattr(h, k, out[k].ctypes.data_as(dp_))
    h.nodecode = out["nodecode"].ctypes.data_as(ip_)
    h.noff = out["noff"].ctypes.data_as(ip_)
    _check(lib.adc_fort67_read(p, C.byref(h)), "adc_fort67_read")
    out.update(im=h.im, it=h.it, timeloc=h.timeloc)
    if h.im != 10:
        del out["ch1"]
    return out
