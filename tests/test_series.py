"""Non-periodic boundary series: the fort.19 elevation and fort.20 normal-flux
files (cstart.F:198-256) and the oracle's restatement of how the reference
steps through them (gwce.F:1659-1674, timestep.F:882-903).

The readers are host code of the library (no GPU).  The known-answer tests
run the oracle: a series that holds one value for every record must give,
bit for bit, the run of a constant periodic forcing of that value (zero
frequency, unit nodal factor, zero phases), since RampElev*(E + r*(E - E))
and E*(FF*RampElev)*cos(0) are the same IEEE products; and the boundary
elevations of a varying series must be the linear interpolation between the
two records the reference holds at each step.
"""
import numpy as np
import pytest

from adcirc_b200 import adcirc_io, model


def _write(path, text):
    path.write_text(text)
    return path


def test_fort19_round_trip(lib, tmp_path):
    rng = np.random.default_rng(5)
    s = model.Series(900.0, rng.normal(size=(7, 5)))
    p = tmp_path / "fort.19"
    adcirc_io.write_fort19(p, s)
    r = adcirc_io.read_fort19(p, 5)
    assert r.interval == 900.0
    assert np.array_equal(r.values, s.values)


def test_fort19_list_directed(lib, tmp_path):
    """One READ per value: extra items on a line are skipped, blank lines
    skipped, Fortran D exponents read; a trailing partial record is an
    error, trailing blank lines are not."""
    p = _write(tmp_path / "fort.19", "600.0  ! ETIMINC\n1.0 99\n\n2.0d0\n3.0\n4.5E-1\n\n\n")
    r = adcirc_io.read_fort19(p, 2)
    assert r.interval == 600.0
    assert np.array_equal(r.values, [[1.0, 2.0], [3.0, 0.45]])
    bad = _write(tmp_path / "bad.19", "600.0\n1\n2\n3\n")
    with pytest.raises(OSError, match="incomplete"):
        adcirc_io.read_fort19(bad, 2)
    with pytest.raises(OSError, match="cannot open"):
        adcirc_io.read_fort19(tmp_path / "missing.19", 2)
    with pytest.raises(OSError, match="increment"):
        adcirc_io.read_fort19(_write(tmp_path / "neg.19", "-5\n1\n2\n3\n4\n"), 2)


def test_fort20_entries(lib, tmp_path):
    """Records take one value per entry of code 2/12/22 and two (flux and
    elevation) per entry of code 32, in LBCODEI order; other entries read
    nothing and hold 0."""
    lbc = np.array([0, 2, 2, 30, 32, 22, 0], np.int32)
    txt = "3600.\n1.5\n2.5\n-0.5 0.25\n7\n" "1.6\n2.6\n-0.6, 0.35\n8\n"
    s = adcirc_io.read_fort20(_write(tmp_path / "fort.20", txt), lbc)
    assert s.interval == 3600.0
    assert np.array_equal(s.values, [[0, 1.5, 2.5, 0, -0.5, 7, 0], [0, 1.6, 2.6, 0, -0.6, 8, 0]])
    assert np.array_equal(s.values2, [[0, 0, 0, 0, 0.25, 0, 0], [0, 0, 0, 0, 0.35, 0, 0]])
    p = tmp_path / "w.20"
    adcirc_io.write_fort20(p, s, lbc)
    r = adcirc_io.read_fort20(p, lbc)
    assert np.array_equal(r.values, s.values) and np.array_equal(r.values2, s.values2)
    with pytest.raises(OSError, match="no boundary entry"):
        adcirc_io.read_fort20(p, np.array([0, 30, 52], np.int32))


def _run(orc, case, n):
    om = orc.OracleModel(case)
    its = om.run(1, n)
    om.close()
    return its


def test_constant_elevation_series_equals_constant_tide(orc):
    neta = model.channel_case().sizes["neta"]
    e = 0.2 + 0.1 * np.linspace(0.0, 1.0, neta)
    tide = model.channel_case()
    a = tide.arrays
    for k in ("amig", "per", "face"):
        a[k][:] = 0.0
    a["ff"][:] = 1.0
    a["emo"][0, :] = e
    a["efa"][0, :] = 0.0
    ser = model.channel_case(elev_series=300.0, series_hours=1.0)
    ser.elev_series.values[:] = e[None, :]
    n = 400   # 2000 s: six record changes
    i0, i1 = _run(orc, tide, n), _run(orc, ser, n)
    assert np.array_equal(i0, i1)
    for f in ("eta2", "etas", "uu2", "vv2", "coef"):
        assert np.array_equal(tide.arrays[f], ser.arrays[f]), f


@pytest.mark.parametrize("river_type", [2, 32])
def test_constant_flux_series_equals_constant_flux(orc, river_type):
    per = model.channel_case(river=0.5, river_type=river_type)
    ser = model.channel_case(river=0.5, river_type=river_type, flux_series=300.0, series_hours=1.0)
    assert ser.flux is None and ser.flux_series is not None
    f = per.flux
    ser.flux_series.values[:] = f.qnam[0][None, :]
    if river_type == 32:
        ser.flux_series.values2[:] = f.enam[0][None, :]
    n = 400
    i0, i1 = _run(orc, per, n), _run(orc, ser, n)
    assert np.array_equal(i0, i1)
    for fld in ("eta2", "uu2", "vv2", "qx2", "coef"):
        assert np.array_equal(per.arrays[fld], ser.arrays[fld]), fld


def test_elevation_series_interpolates_records(orc):
    """Boundary ETA2 after every step is RampElev times the interpolation
    between the record pair, the pair moving on when TimeLoc passes the later
    record time (the record times accumulate as ETIME2 = ETIME1 + ETIMINC)."""
    case = model.channel_case(elev_series=150.0, series_hours=1.0)
    s = case.elev_series
    nbd = case.arrays["nbd"] - 1
    om = orc.OracleModel(case)
    t1, t2, k = 0.0, s.interval, 0
    moves = 0
    for it in range(1, 301):
        om.step(it)
        st = case.schedule.step(it)
        if st.timeloc > t2:
            t1 = t2
            t2 = t1 + s.interval
            k += 1
            moves += 1
        r = (st.timeloc - t1) / s.interval
        e1, e2 = s.values[k], s.values[k + 1]
        want = st.rampelev * (e1 + r * (e2 - e1))
        # ETA2 = ETAS + ETA1 after the solve (gwce.F:2006-2008): equal to
        # rounding; another record pair or ratio would be off by far more
        assert np.allclose(case.arrays["eta2"][nbd], want, rtol=1e-12, atol=1e-15), it
    om.close()
    assert moves == 9


def test_series_end_stops_the_run(orc):
    case = model.channel_case(elev_series=600.0, series_hours=0.25)   # records to 1800 s
    om = orc.OracleModel(case)
    om.run(1, 360)   # TimeLoc 1800 s: the last pair still holds
    with pytest.raises(RuntimeError, match="status"):
        om.step(361)
    om.close()
