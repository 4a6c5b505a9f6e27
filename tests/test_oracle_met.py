"""CPU checks of the oracle's NWS = 8 vortex forcing (HollandGet,
nws08.F90:562-717, and the stress of wind.F:1172-1198).

The reference ships no wind fixtures for this path, so the restatement is
pinned by an independent numpy evaluation of the same formulas and by
known answers of the Holland profile: p(RMW) = pc + dp/e, the pressure
minimum at the node nearest the eye, background pressure far away, the
wind maximum near RMW, and GetHollandStormData's track bookkeeping.
"""
import math

import numpy as np
import pytest

G = 9.80665


def _holland_numpy(case, v, lon, lat, wt, timeloc, rampmete):
    """Independent numpy evaluation of the per-node vortex (same operation
    order as nws08.F90:642-715 and wind.F:1174-1193)."""
    f = v.fixes
    a = case.arrays
    i = np.searchsorted(f[:, 0], timeloc)   # first fix with time >= timeloc
    cp = f[i - 1, 3] + wt * (f[i, 3] - f[i - 1, 3])
    spd = f[i - 1, 4] + wt * (f[i, 4] - f[i - 1, 4])
    rmw = f[i - 1, 5] + wt * (f[i, 5] - f[i - 1, 5])
    tvx = f[i - 1, 6] + wt * (f[i, 6] - f[i - 1, 6])
    tvy = f[i - 1, 7] + wt * (f[i, 7] - f[i - 1, 7])
    dp = max(1013.0 * 100.0 - cp, 100.0)
    spd = (spd - math.sqrt(tvx * tvx + tvy * tvy)) / v.bladj
    b = min(max(v.rho_air * 2.718281828459045 * (spd * spd) / dp, 1.0), 2.5)
    rmw *= 1000.0
    dx, dy = a["x"] - lon, a["y"] - lat
    th = np.arctan2(dy, dx)
    rad = np.sqrt(dx * dx + dy * dy)
    cf = a["corif"]
    al = (rmw / rad) ** b
    pr = cp + dp * np.exp(-al)
    vr = np.sqrt(al * np.exp(1.0 - al) * spd * spd + 0.25 * (rad * rad) * (cf * cf)) - 0.5 * rad * np.abs(cf)
    vr = vr * v.wind_mult * v.bladj
    wx = -vr * np.sin(th) + (np.abs(vr) / spd) * tvx
    wy = vr * np.cos(th) + (np.abs(vr) / spd) * tvy
    wx, wy = wx * 0.8928, wy * 0.8928
    pr = np.clip(pr, 0.85e5, 1.1e5)
    wx, wy = np.clip(wx, -200, 200), np.clip(wy, -200, 200)
    prn = pr / (1000.0 * G)
    mag = np.sqrt(wx * wx + wy * wy)
    drag = np.minimum(0.001 * (0.75 + 0.067 * mag), v.drag_limit)
    awr = v.rho_air / 1000.0
    pb = case.params["prbckgrnd_mh2o"]
    return (rampmete * awr * drag * wx * mag, rampmete * awr * drag * wy * mag,
            pb + rampmete * (prn - pb), rmw, cp, dp, b)


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_vortex_fields_match_numpy(orc):
    from adcirc_b200 import model
    case = model.channel_case(vortex=True)
    v = case.vortex
    m = orc.OracleModel(case)
    sch = case.schedule
    # step 1: position from the default WTRATIO = 1 (the later fix), then
    # step 2: position from step 1's WTRATIO (nws08.F90:856-857)
    f = v.fixes
    for it, lonlat_wt in ((1, 1.0), (2, None)):
        s = sch.step(it)
        assert m.met(it) == 0
        if lonlat_wt is None:
            lonlat_wt = (sch.step(1).timeloc - f[0, 0]) / (f[1, 0] - f[0, 0])
        lon = f[0, 1] + lonlat_wt * (f[1, 1] - f[0, 1])
        lat = f[0, 2] + lonlat_wt * (f[1, 2] - f[0, 2])
        wt = (s.timeloc - f[0, 0]) / (f[1, 0] - f[0, 0])
        wsx, wsy, pr2, *_ = _holland_numpy(case, v, lon, lat, wt, s.timeloc, s.rampmete)
        a = case.arrays
        assert _rel(a["wsx2"], wsx) < 1e-12
        assert _rel(a["wsy2"], wsy) < 1e-12
        assert _rel(a["pr2"], pr2) < 1e-14
    m.close()


def test_holland_profile_known_answers(orc):
    """Pressure equals pc + dp/e at r = RMW, is lowest at the node nearest
    the eye and tends to the background far away; the wind peaks near RMW."""
    from adcirc_b200 import model
    case = model.channel_case(vortex=True)
    v = case.vortex
    f = v.fixes
    lon, lat = f[0, 1], f[0, 2]   # the eye inside the channel
    s = case.schedule.step(1)
    wt = (s.timeloc - f[0, 0]) / (f[1, 0] - f[0, 0])
    wsx, wsy, pr2, rmw, cp, dp, b = _holland_numpy(case, v, lon, lat, wt, s.timeloc, 1.0)
    # the analytic profile at r = RMW
    p_rmw = cp + dp * math.exp(-1.0)
    assert 0.85e5 < p_rmw < 1.1e5
    a = case.arrays
    r = np.hypot(a["x"] - lon, a["y"] - lat)
    # inside ~RMW/10 exp(-alpha) underflows against pc, so several nodes tie
    assert pr2[np.argmin(r)] == pr2.min()
    pb = case.params["prbckgrnd_mh2o"]
    far = r > 20 * rmw
    if far.any():
        assert np.all(np.abs(pr2[far] - pb) < 0.05 * dp / (1000.0 * G))
    mag = np.hypot(wsx, wsy)
    ring = (r > 0.6 * rmw) & (r < 1.6 * rmw)
    assert mag[ring].max() >= mag[r < 0.3 * rmw].max()
    assert 1.0 <= b <= 2.5 and abs(b - 1.3) < 1e-9


def test_vortex_track_bookkeeping(orc):
    from adcirc_b200 import model
    case = model.channel_case(vortex=True)
    v = case.vortex
    # a track that ends 12 s after the start: the third step passes it
    short = model.Vortex(v.fixes[:2].copy())
    short.fixes[1, 0] = 12.0
    m = orc.OracleModel(case)
    m.set_vortex(short)
    assert m.met(1) == 0 and m.met(2) == 0
    assert m.met(3) != 0          # nws08.F90:847-852 terminates here
    # invalid tracks
    bad = model.Vortex(v.fixes[:1].copy())
    with pytest.raises(ValueError):
        m.set_vortex(bad)
    rev = model.Vortex(v.fixes[::-1].copy())
    with pytest.raises(ValueError):
        m.set_vortex(rev)
    late = model.Vortex(v.fixes.copy(), start_time=1e9)
    with pytest.raises(ValueError):
        m.set_vortex(late)
    m.close()


def calm_track_case(**kw):
    """The channel with a vortex track of fixes every 100 s whose third fix
    (t = 200 s) is a CALM line: steps with 100 s < TimeLoc <= 300 s have a
    CALM fix on one side of them."""
    from adcirc_b200 import model
    case = model.channel_case(vortex=True, **kw)
    case.vortex = model.straight_track(30.3e3, 3.7e3, 80.0, 6.0, 960.0, 8.0, 1.3, hours=1.0,
                                       interval_h=100.0 / 3600.0)
    case.vortex.fixes[2, 3] = -99999.0
    return case


def test_vortex_calm_period(orc):
    """While a CALM line brackets the time, HollandGet returns no wind and
    the background pressure in metres of water (nws08.F90:588-601), so the
    stress is zero and PR2 the ramped background; the storm is back after
    it."""
    case = calm_track_case()
    m = orc.OracleModel(case)
    a = case.arrays
    pb = case.params["prbckgrnd_mh2o"]
    g = case.params["g"]
    for it in range(1, 80):
        m.step(it)
        st = case.schedule.step(it)
        calm = 100.0 < st.timeloc <= 300.0
        if calm:
            assert not np.any(a["wsx2"]) and not np.any(a["wsy2"]), it
            want = pb + st.rampmete * (1013.0 * 100.0 / (1000.0 * g) - pb)
            assert np.all(a["pr2"] == want), it
        elif st.timeloc > 300.0:
            assert np.abs(a["wsx2"]).max() > 0.0, it
    m.close()


def test_surge_track_makes_landfall():
    """The surge case's track (pc 940 hPa, Rmax 40 km, B 1.3, 5 m/s) starts
    offshore and crosses the coast (y ~ 640 km) within the simulated day."""
    from adcirc_b200 import model
    v = model.straight_track(501234.5, 300678.9, 90.0, 5.0, 940.0, 40.0, 1.3, hours=30.0)
    f = v.fixes
    assert np.allclose(f[:, 3], 94000.0) and np.allclose(f[:, 5], 40.0)
    y_day = np.interp(86400.0, f[:, 0], f[:, 2])
    assert f[0, 2] < 600e3 < y_day
    dp = 101300.0 - 94000.0
    spd = (f[0, 4] - 5.0) / v.bladj
    assert abs(v.rho_air * math.e * spd * spd / dp - 1.3) < 1e-12
