"""fort.22 reader for NWS = 8 (adc_fort22_read; readBestTrackData,
nws08.F90:884-1098).  The lines are made here, for an invented storm, in the
fixed columns of the reference's FORMAT 228; the expected fixes are worked
out independently with numpy (TIMECONV days, the CPP projection, the
reference's unit factors and the haversine translation speed of uvtrans)."""
import math

import numpy as np
import pytest

from adcirc_b200 import adcirc_io, model

R = 6378206.4
D2R = math.pi / 180.0
NM = 1.852000003180799
KT = 0.51444444


def atcf(yr, mo, dy, hr, typ, inc, lat10, lon10, spd, cp, rrp, rmw, ns="N", ew="W"):
    """One line with the FORMAT 228 fields at their columns: date at 9-18,
    type 25-28, forecast hour 31-33, latitude 35-39, longitude 42-46, Vmax
    49-51, central pressure 54-57, closed-isobar radius 105-107 and Rmax
    110-112; the rest is filler of commas and letters."""
    s = "ZZ, 99, " + f"{yr:04d}{mo:02d}{dy:02d}{hr:02d}" + ",   , " + f"{typ:<4s}" + ", "
    s += f"{inc:3d}" + "," + f"{lat10:4d}" + ns + ", " + f"{lon10:4d}" + ew + ", "
    s += f"{spd:3d}" + ", " + f"{cp:4d}"
    s += (", XX,  34, NEQ,    0,    0,    0,    0, 1010,   ").ljust(47)[:47]
    s += f"{rrp:3d}" + ", " + f"{rmw:3d}" + ",   0,   0,   L,   0,    ,   0,   0,  NONAME, D,"
    assert s[24:28] == f"{typ:<4s}" and s[104:107] == f"{rrp:3d}" and s[109:112] == f"{rmw:3d}"
    return s


LINES = [
    atcf(2001, 2, 28, 18, "BEST", 0, 251, 802, 45, 990, 200, 30),
    atcf(2001, 2, 28, 18, "BEST", 0, 251, 802, 45, 990, 180, 30),   # repeated time: dropped
    atcf(2001, 3, 1, 0, "BEST", 0, 257, 811, 55, 981, 210, 25),
    atcf(2001, 3, 1, 6, "BEST", 0, 266, 819, 70, 968, 220, 20),
    atcf(2001, 3, 1, 6, "OFCL", 0, 266, 819, 70, 968, 220, 20),     # coincides: dropped
    atcf(2001, 3, 1, 6, "OFCL", 12, 280, 830, 80, 960, 230, 18),
    atcf(2001, 3, 1, 6, "OFCL", 12, 281, 830, 80, 960, 230, 18),    # same increment: dropped
    atcf(2001, 3, 1, 6, "CALM", 24, 295, 842, 0, 0, 0, 0),
    atcf(2001, 3, 1, 6, "OFCL", 36, 310, 851, 50, 985, 240, 35),
]
REF = dict(irefyr=2001, irefmo=2, irefday=28, irefhr=12)   # six hours before the first fix


def _write(tmp_path, lines, name="fort.22"):
    p = tmp_path / name
    p.write_text("\n".join(lines) + "\n")
    return p


def _haversine(dx, dy, y1, y2):
    return R * 2.0 * math.asin(math.sqrt(math.sin(dy / 2) ** 2 +
                                         math.cos(y1 * D2R) * math.cos(y2 * D2R) * math.sin(dx / 2) ** 2))


def test_fort22_track(lib, tmp_path):
    v = adcirc_io.read_fort22(_write(tmp_path, LINES), slam0=-81.0, sfea0=27.0, bladj=0.9, **REF)
    f = v.fixes
    assert f.shape == (6, 8)
    # TIMECONV: 2001 is not divisible by 4, so 1 March 00 h follows 28 February
    # 18 h by 6 h; the forecasts add 12 h and then their increment changes
    hours = np.array([6, 12, 18, 30, 42, 54])
    assert np.array_equal(f[:, 0], hours * 3600.0)
    lat = np.array([25.1, 25.7, 26.6, 28.0, 29.5, 31.0])
    lon = -np.array([80.2, 81.1, 81.9, 83.0, 84.2, 85.1])
    assert np.allclose(f[:, 1], R * math.cos(27.0 * D2R) * (lon * D2R + 81.0 * D2R), rtol=1e-14)
    assert np.allclose(f[:, 2], R * (lat * D2R), rtol=1e-14)
    assert np.array_equal(f[:, 3], [99000.0, 98100.0, 96800.0, 96000.0, -99999.0, 98500.0])
    assert np.allclose(f[:, 4], np.array([45, 55, 70, 80, 0, 50]) * KT, rtol=1e-15)
    assert np.allclose(f[:, 5], np.array([30, 25, 20, 18, 0, 35]) * NM, rtol=1e-15)
    for i in range(1, 6):
        avg = (lat[i - 1] + lat[i]) / 2
        dt = f[i, 0] - f[i - 1, 0]
        u = _haversine((lon[i] - lon[i - 1]) * D2R, 0.0, avg, avg) / dt
        w = _haversine(0.0, (lat[i] - lat[i - 1]) * D2R, lat[i - 1], lat[i]) / dt
        assert math.isclose(f[i, 6], -u, rel_tol=1e-13)   # moving west
        assert math.isclose(f[i, 7], w, rel_tol=1e-13)
    assert f[0, 6] == f[1, 6] and f[0, 7] == f[1, 7]
    assert v.bladj == 0.9


def test_fort22_leap_year_and_hemispheres(lib, tmp_path):
    lines = [atcf(2004, 2, 28, 0, "BEST", 0, 100, 1500, 40, 995, 150, 20, ns="S", ew="E"),
             atcf(2004, 3, 1, 0, "BEST", 0, 120, 1490, 45, 990, 150, 20, ns="S", ew="E")]
    v = adcirc_io.read_fort22(_write(tmp_path, lines), 2004, 2, 28, 0)
    assert np.array_equal(v.fixes[:, 0], [0.0, 2 * 86400.0])   # 29 February exists
    assert v.fixes[1, 2] < v.fixes[0, 2] < 0.0                  # southern, moving south
    assert v.fixes[1, 6] < 0.0 and v.fixes[1, 7] < 0.0


def test_fort22_errors(lib, tmp_path):
    with pytest.raises(OSError, match="BEST, OFCL or CALM"):
        adcirc_io.read_fort22(_write(tmp_path, LINES[:3] + [LINES[3].replace("BEST", "CARQ")]), **REF)
    no_rmw = atcf(2001, 3, 1, 6, "OFCL", 12, 280, 830, 80, 960, 230, 0)
    with pytest.raises(OSError, match="Rmax"):
        adcirc_io.read_fort22(_write(tmp_path, LINES[:4] + [no_rmw]), **REF)
    with pytest.raises(OSError, match="before RNDAY"):
        adcirc_io.read_fort22(_write(tmp_path, LINES), rnday=3.0, **REF)
    with pytest.raises(OSError, match="cannot open"):
        adcirc_io.read_fort22(tmp_path / "none.22", **REF)
    assert adcirc_io.read_fort22(_write(tmp_path, LINES), rnday=2.0, **REF).fixes.shape[0] == 6


def test_fort22_track_drives_the_oracle(orc, tmp_path):
    """A track read from a fort.22 drives the oracle's vortex step."""
    lines = [atcf(2001, 6, 1, 0, "BEST", 0, 0, 0, 60, 970, 200, 8, ew="E"),
             atcf(2001, 6, 1, 6, "BEST", 0, 3, 2, 60, 968, 200, 8, ew="E")]
    v = adcirc_io.read_fort22(_write(tmp_path, lines), 2001, 6, 1, 0, bladj=0.9)
    case = model.channel_case(vortex=True)
    case.vortex = v
    m = orc.OracleModel(case)
    m.run(1, 20)
    m.close()
    assert np.abs(case.arrays["wsx2"]).max() > 0.0
