"""ADCIRC text files at the edges of the hot path, through libadcgpu's host
functions: fort.14 meshes (read14, mesh.F:319-581) and the full-domain
ASCII outputs fort.63/fort.64 (globalio.F:544-643, 802-930, 1005-1085)."""
from __future__ import annotations

import ctypes as C
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
    segs, q = [], 0
    for k in range(nbou):
        segs.append((int(ibtype[k]), nbvv[q:q + nvell[k]].astype(np.int64) - 1))
        q += int(nvell[k])
    name = title.value.decode(errors="replace").strip() or os.path.basename(os.fsdecode(path))
    meta = {"lx": float(x.max() - x.min()), "ly": float(y.max() - y.min()),
            "open_segments": [int(v) for v in nvdll[:nope]], "source": os.fsdecode(path)}
    return RawMesh(name, x, y, dp, np.asarray(nm, np.int64) - 1,
                   nbdv[:neta].astype(np.int64) - 1, segs, meta)


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
    _check(lib.adc_fort14_write(os.fsencode(path), (title or raw.name).encode()[:80],
                                int(x.size), int(nm.shape[0]), ptr(x, dp_), ptr(y, dp_),
                                ptr(dp, dp_), ptr(nm, ip_), len(lens), ptr(nvdll, ip_),
                                ptr(nbdv, ip_), len(raw.land_segments), ptr(nvell, ip_),
                                ptr(ibtype, ip_), ptr(nbvv, ip_)), "adc_fort14_write")


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
