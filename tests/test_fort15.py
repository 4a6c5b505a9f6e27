"""fort.15 reader and writer (csrc/fort15_io.cpp, adcirc_io.read_fort15 /
write_fort15, model.case_from_files): the record order of READ_INPUT
(read_input.F:949-4566), round trips through files, and a case built from
files against the same case built directly.  No GPU."""
import math

import numpy as np
import pytest

from adcirc_b200 import _lib, adcirc_io, model

# A hand-written 2DDI fort.15 in the layout read_input reads: annotations
# after the values, a comma-separated record, a D exponent, NRAMP = 2,
# NOLIFA = 2 (H0 record with the two integers), hybrid friction, two
# elevation constituents on a 3-node open boundary, stations, one harmonic
# analysis constituent and the two namelists the path uses.
HAND = """Hand-written test run
test-1
1                ! NFOVER
0                ! NABOUT
0                ! NSCREEN
0                ! IHOT
1                ! ICS
0                ! IM
2                ! NOLIBF
2                ! NOLIFA
1                ! NOLICA
0                ! NOLICAT
0                ! NWP
0                ! NCOR
0                ! NTIP
0                ! NWS
2                ! NRAMP
9.81             ! G
-1.0             ! TAU0
2.0              ! DTDP
0.25             ! STATIM
0.0              ! REFTIM
3.5              ! RNDAY
0.75, 0.1, 0.0   ! DRAMP, DRAMPExtFlux, FluxSettlingTime
0.35 0.30 0.35   ! A00, B00, C00
0.08 5 7 0.02    ! H0, NODEDRYMIN, NODEWETMIN, VELMIN
-90.0 30.0       ! SLAM0, SFEA0
0.003 1.5 10.0 0.3333333333333333   ! CF, HBREAK, FTHETA, FGAMMA
12.5             ! ESLM
7.29D-5          ! CORI
0                ! NTIF
2                ! NBFR
M2
0.000140518902509 1.0 30.0
K1
0.0000729211583579 0.98 -45.0
M2
0.5 10.0
0.6 20.0
0.7 30.0
K1
0.2 0.0
0.25 90.0
0.3 180.0
100.0            ! ANGINN
1 0.5 3.5 180    ! NOUTE, TOUTSE, TOUTFE, NSPOOLE
2                ! NSTAE
1000.0 2000.0 gauge A
3000.5 4000.25
0 0.0 0.0 0      ! NOUTV, TOUTSV, TOUTFV, NSPOOLV
0                ! NSTAV
1 0.5 3.5 720    ! NOUTGE, TOUTSGE, TOUTFGE, NSPOOLGE
0 0.0 0.0 0      ! NOUTGV, TOUTSGV, TOUTFGV, NSPOOLGV
1                ! NFREQ
M2
0.000140518902509 1.0 0.0
1.0 3.5 10 0.5   ! THAS, THAF, NHAINC, FMV
1 0 1 0          ! NHASE, NHASV, NHAGE, NHAGV
0 0              ! NHSTAR, NHSINC
1 0 1.0E-10 25   ! ITITER, ISLDIA, CONVCR, ITMAX
&wetDryControl outputNodeCode=.false., slim = 2.5E-4 /
&metControl WindDragLimit=0.0025, DragLawString='Garratt' /
"""


def _write(tmp_path, text, name="fort.15"):
    p = tmp_path / name
    p.write_text(text)
    return p


def test_hand_written_fort15(lib, tmp_path):
    f = adcirc_io.read_fort15(_write(tmp_path, HAND), 3, [])
    assert f.p.rundes.decode() == "Hand-written test run" and f.p.runid.decode() == "test-1"
    assert (f.nolibf, f.nolifa, f.nolica, f.nolicat, f.nramp, f.nws) == (2, 2, 1, 0, 2, 0)
    assert (f.g, f.tau0, f.dtdp, f.statim, f.rnday) == (9.81, -1.0, 2.0, 0.25, 3.5)
    # NRAMP = 2: DRamp, DRampExtFlux, FluxSettlingTime; the other ramps take DRamp
    assert (f.dramp, f.dramp_extflux, f.flux_settling_time) == (0.75, 0.1, 0.0)
    assert f.dramp_elev == f.dramp_mete == f.dramp_intflux == f.dramp_tip == 0.75
    assert (f.h0, f.nodedrymin, f.nodewetmin, f.velmin) == (0.08, 5, 7, 0.02)
    assert (f.cf, f.hbreak, f.ftheta, f.fgamma) == (0.003, 1.5, 10.0, 0.3333333333333333)
    assert (f.eslm, f.cori, f.anginn) == (12.5, 7.29e-5, 100.0)
    assert f.bountag == ["M2", "K1"]
    assert np.array_equal(f.amig, [0.000140518902509, 0.0000729211583579])
    assert np.allclose(f.face, np.deg2rad([30.0, -45.0]), rtol=1e-15, atol=0)
    assert np.array_equal(f.emo, [[0.5, 0.6, 0.7], [0.2, 0.25, 0.3]])
    assert np.allclose(f.efa, np.deg2rad([[10.0, 20.0, 30.0], [0.0, 90.0, 180.0]]), rtol=1e-15, atol=0)
    assert (f.oute.nout, f.oute.touts, f.oute.toutf, f.oute.nspool) == (1, 0.5, 3.5, 180)
    assert f.nstae == 2 and np.array_equal(f.xel, [1000.0, 3000.5]) and np.array_equal(f.yel, [2000.0, 4000.25])
    assert f.outge.nspool == 720 and f.nfreq == 1 and f.namefr == ["M2"]
    assert (f.thas, f.thaf, f.nhainc, f.fmv) == (1.0, 3.5, 10, 0.5)
    assert (f.ititer, f.isldia, f.convcr, f.itmax) == (1, 0, 1.0e-10, 25)
    assert f.has_slim and f.slim == 2.5e-4
    assert f.has_wind_drag_limit and f.wind_drag_limit == 0.0025


def test_fort15_write_read_round_trip(lib, tmp_path):
    f = adcirc_io.read_fort15(_write(tmp_path, HAND), 3, [])
    out = tmp_path / "again.15"
    adcirc_io.write_fort15(out, f, 3, [])
    g = adcirc_io.read_fort15(out, 3, [])
    for name, _ in _lib.AdcFort15._fields_:
        a, b = getattr(f.p, name), getattr(g.p, name)
        if isinstance(a, _lib.AdcOutputSpec):
            a, b = (a.nout, a.nspool, a.touts, a.toutf), (b.nout, b.nspool, b.touts, b.toutf)
        if name == "nwp":
            continue   # attribute names are not written
        assert a == b, name
    for k, v in f.tables.items():
        if k in ("face", "efa", "fface", "qnph", "enph", "facet"):   # degrees in the file
            assert np.allclose(v, g.tables[k], rtol=2e-16, atol=1e-300), k
        else:
            assert np.array_equal(v, g.tables[k]), k


def test_case_from_files_equals_the_built_case(lib, orc, tmp_path):
    """The river channel written as fort.14 + fort.15 and read back: the
    same bound arrays, parameters and flux, and the oracle steps both to
    the same state."""
    import oracle
    c = model.channel_case(river=1.5)
    adcirc_io.write_fort14(c.meta["raw"], tmp_path / "fort.14")
    adcirc_io.write_fort15(tmp_path / "fort.15", model.fort15_for_case(c), c.sizes["neta"],
                           c.arrays["lbcodei"][:c.sizes["nvel"]])
    c2 = model.case_from_files(tmp_path / "fort.14", tmp_path / "fort.15")
    assert c2.params == c.params
    for k, v in c.arrays.items():
        assert np.array_equal(v, c2.arrays[k]), k
    assert np.array_equal(c.flux.qnam, c2.flux.qnam) and np.array_equal(c.flux.famig, c2.flux.famig)
    its = []
    for case in (c, c2):
        om = oracle.OracleModel(case)
        its.append(om.run(1, 30))
        om.close()
    assert np.array_equal(its[0], its[1])
    assert np.array_equal(c.arrays["eta2"], c2.arrays["eta2"])
    assert np.array_equal(c.arrays["uu2"], c2.arrays["uu2"])


def test_case_from_files_surge_settings(lib, tmp_path):
    """Hybrid friction, the slope limiter, TAU0 = -1 and two constituents
    survive the files (a small graded mesh of the surge family)."""
    from adcirc_b200 import meshgen
    raw = meshgen.surge_mesh(seed=11, target_nodes=6000, alpha=0.6)
    raw.meta = {k: v for k, v in raw.meta.items() if k != "coast_fn"}
    c = model.surge_case(raw=raw, vortex=False)
    adcirc_io.write_fort14(c.meta["raw"], tmp_path / "fort.14")
    adcirc_io.write_fort15(tmp_path / "fort.15", model.fort15_for_case(c), c.sizes["neta"],
                           c.arrays["lbcodei"][:c.sizes["nvel"]])
    c2 = model.case_from_files(tmp_path / "fort.14", tmp_path / "fort.15")
    assert c2.params == c.params
    for k, v in c.arrays.items():
        if k == "efa":
            assert np.allclose(v, c2.arrays[k], rtol=2e-16, atol=0), k
        else:
            assert np.array_equal(v, c2.arrays[k]), k


def _lines(text):
    return text.splitlines(keepends=True)


@pytest.mark.parametrize("edit, code, what", [
    (lambda L: L[:7] + ["1   ! IM\n"] + L[8:], -6, "IM"),
    (lambda L: L[:15] + ["12  ! NWS\n"] + L[16:], -6, "NWS"),
    (lambda L: L[:30], -1, "record"),
    (lambda L: L[:29] + ["seven  ! CORI\n"] + L[30:], -1, "CORI"),
    (lambda L: [ln.replace("2                ! NSTAE", "-2               ! NSTAE") for ln in L], -6, "151"),
])
def test_fort15_errors(lib, tmp_path, edit, code, what):
    p = _write(tmp_path, "".join(edit(_lines(HAND))))
    o = _lib.AdcFort15()
    rc = lib.adc_fort15_read(str(p).encode(), 3, 0, None, o, None)
    assert rc == code
    assert what in _lib.last_error()


def test_case_from_files_refuses_uncovered_runs(lib, tmp_path):
    c = model.channel_case()
    adcirc_io.write_fort14(c.meta["raw"], tmp_path / "fort.14")
    f = model.fort15_for_case(c)
    f.p.ics = 2
    f.p.ncor = 1
    adcirc_io.write_fort15(tmp_path / "fort.15", f, c.sizes["neta"], c.arrays["lbcodei"][:c.sizes["nvel"]])
    with pytest.raises(NotImplementedError, match="ICS = 2.*NCOR = 1"):
        model.case_from_files(tmp_path / "fort.14", tmp_path / "fort.15")


def test_river_radiation_case_through_files(lib, orc, tmp_path):
    """IBTYPE 52 with a flux settling time: NRAMP, FluxSettlingTime and the
    river flux records survive the files, and the oracle steps both cases
    (through the settling and after it) to the same state."""
    import oracle
    c = model.channel_case(river=0.5, river_type=52, flux_settling=0.02)
    adcirc_io.write_fort14(c.meta["raw"], tmp_path / "fort.14")
    adcirc_io.write_fort15(tmp_path / "fort.15", model.fort15_for_case(c), c.sizes["neta"],
                           c.arrays["lbcodei"][:c.sizes["nvel"]])
    c2 = model.case_from_files(tmp_path / "fort.14", tmp_path / "fort.15")
    assert c2.flux.flux_settling_it == c.flux.flux_settling_it == 345
    assert c2.schedule.flux_settling_time == c.schedule.flux_settling_time
    for k, v in c.arrays.items():
        assert np.array_equal(v, c2.arrays[k]), k
    for case in (c, c2):
        om = oracle.OracleModel(case)
        om.run(1, 500)
        om.close()
    assert np.array_equal(c.arrays["eta2"], c2.arrays["eta2"])


def test_coupled_flux_radiation_case_through_files(lib, orc, tmp_path):
    """IBTYPE 32: the four-item flux records (QNAM, QNPH, ENAM, ENPH)
    survive the files, and the oracle steps both cases to the same state."""
    import oracle
    c = model.channel_case(river=0.5, river_type=32, river_eta=0.07)
    adcirc_io.write_fort14(c.meta["raw"], tmp_path / "fort.14")
    adcirc_io.write_fort15(tmp_path / "fort.15", model.fort15_for_case(c), c.sizes["neta"],
                           c.arrays["lbcodei"][:c.sizes["nvel"]])
    c2 = model.case_from_files(tmp_path / "fort.14", tmp_path / "fort.15")
    assert np.array_equal(c.flux.enam, c2.flux.enam) and np.array_equal(c.flux.qnam, c2.flux.qnam)
    for k, v in c.arrays.items():
        assert np.array_equal(v, c2.arrays[k]), k
    for case in (c, c2):
        om = oracle.OracleModel(case)
        om.run(1, 300)
        om.close()
    assert np.array_equal(c.arrays["eta2"], c2.arrays["eta2"])


def test_series_case_through_files(lib, orc, tmp_path):
    """NBFR 0 with a fort.19 beside the fort.15, and NFFR 0 with a fort.20:
    case_from_files finds both as the reference does (read_input.F:1893-1898,
    cstart.F:198-256), the records survive the files, and the oracle steps
    both cases to the same state."""
    import oracle
    c = model.channel_case(river=0.5, elev_series=150.0, flux_series=300.0, series_hours=1.0)
    lbc = c.arrays["lbcodei"][:c.sizes["nvel"]]
    adcirc_io.write_fort14(c.meta["raw"], tmp_path / "fort.14")
    adcirc_io.write_fort15(tmp_path / "fort.15", model.fort15_for_case(c), c.sizes["neta"], lbc)
    adcirc_io.write_fort19(tmp_path / "fort.19", c.elev_series)
    adcirc_io.write_fort20(tmp_path / "fort.20", c.flux_series, lbc)
    c2 = model.case_from_files(tmp_path / "fort.14", tmp_path / "fort.15")
    assert c2.flux is None and c2.sizes["nbfr"] == 0
    assert np.array_equal(c2.elev_series.values, c.elev_series.values)
    assert np.array_equal(c2.flux_series.values, c.flux_series.values)
    assert c2.elev_series.interval == 150.0 and c2.flux_series.interval == 300.0
    for case in (c, c2):
        om = oracle.OracleModel(case)
        om.run(1, 200)
        om.close()
    assert np.array_equal(c.arrays["eta2"], c2.arrays["eta2"])
    assert np.array_equal(c.arrays["uu2"], c2.arrays["uu2"])


def test_vortex_case_through_files(lib, orc, tmp_path):
    """NWS = 8: the track comes from the fort.22 beside the fort.15, read
    against the fort.15's wind reference time and projection centre."""
    import oracle
    from test_fort22 import atcf
    c = model.channel_case(vortex=True)
    lbc = c.arrays["lbcodei"][:c.sizes["nvel"]]
    adcirc_io.write_fort14(c.meta["raw"], tmp_path / "fort.14")
    adcirc_io.write_fort15(tmp_path / "fort.15", model.fort15_for_case(c), c.sizes["neta"], lbc)
    lines = [atcf(2000, 1, 1, 0, "BEST", 0, 0, 0, 60, 970, 200, 8, ew="E"),
             atcf(2000, 1, 1, 6, "BEST", 0, 2, 3, 60, 968, 200, 8, ew="E"),
             atcf(2000, 1, 2, 0, "BEST", 0, 5, 6, 55, 975, 200, 9, ew="E")]
    (tmp_path / "fort.22").write_text("\n".join(lines) + "\n")
    with pytest.raises(NotImplementedError, match="fort.22"):
        model.case_from_files(tmp_path / "fort.14", tmp_path / "fort.15", fort22=tmp_path / "none")
    c2 = model.case_from_files(tmp_path / "fort.14", tmp_path / "fort.15")
    want = adcirc_io.read_fort22(tmp_path / "fort.22", 2000, 1, 1, 0)
    assert np.array_equal(c2.vortex.fixes, want.fixes)
    assert c2.vortex.bladj == c.vortex.bladj
    om = oracle.OracleModel(c2)
    om.run(1, 20)
    om.close()
    assert np.abs(c2.arrays["wsx2"]).max() > 0.0


def test_external_barrier_case_through_files(lib, orc, tmp_path):
    """An external barrier segment (crest heights and coefficients in the
    fort.14) and DRampIntFlux (NRAMP 8 in the fort.15) survive the files,
    and the oracle steps both cases to the same state."""
    import oracle
    c = model.channel_case(barrier=-0.5, barrier_type=13)
    c.schedule.dramp_intflux = 0.2
    adcirc_io.write_fort14(c.meta["raw"], tmp_path / "fort.14")
    adcirc_io.write_fort15(tmp_path / "fort.15", model.fort15_for_case(c), c.sizes["neta"],
                           c.arrays["lbcodei"][:c.sizes["nvel"]])
    c2 = model.case_from_files(tmp_path / "fort.14", tmp_path / "fort.15")
    assert c2.schedule.dramp_intflux == 0.2
    for k, v in c.arrays.items():
        assert np.array_equal(v, c2.arrays[k]), k
    for case in (c, c2):
        om = oracle.OracleModel(case)
        om.run(1, 200)
        om.close()
    assert np.array_equal(c.arrays["eta2"], c2.arrays["eta2"])


def test_nws08_namelist(lib, tmp_path):
    """&nws08Control (nws08.F90:318-413): WindMultiplier and the averaging
    minute reach the vortex; other vortex models, background winds, B
    calculations and inflow angles are refused."""
    from test_fort22 import atcf
    c = model.channel_case(vortex=True)
    c.vortex.wind_mult, c.vortex.avg_minute = 1.25, 10
    lbc = c.arrays["lbcodei"][:c.sizes["nvel"]]
    adcirc_io.write_fort14(c.meta["raw"], tmp_path / "fort.14")
    f15 = tmp_path / "fort.15"
    adcirc_io.write_fort15(f15, model.fort15_for_case(c), c.sizes["neta"], lbc)
    assert "&nws08Control" in f15.read_text()
    lines = [atcf(2000, 1, 1, 0, "BEST", 0, 0, 0, 60, 970, 200, 8, ew="E"),
             atcf(2000, 1, 2, 0, "BEST", 0, 5, 6, 55, 975, 200, 9, ew="E")]
    (tmp_path / "fort.22").write_text("\n".join(lines) + "\n")
    c2 = model.case_from_files(tmp_path / "fort.14", f15)
    assert c2.vortex.wind_mult == 1.25 and c2.vortex.avg_minute == 10
    text = f15.read_text()
    for bad in ("vortexModel='CLE15'", "backgroundWindModel = 'LC12'", "BCalc='exact'",
                "useInflow=.true.", "thetaLatDep = T"):
        g = tmp_path / "bad.15"
        g.write_text(text.replace("&nws08Control ", f"&nws08Control {bad}, "))
        o = _lib.AdcFort15()
        rc = lib.adc_fort15_read(str(g).encode(), c.sizes["neta"], int(lbc.size),
                                 lbc.ctypes.data_as(_lib.ip_), o, None)
        assert rc == _lib.ADC_ERR_UNSUPPORTED, bad
        assert bad.split("=")[0].strip() in _lib.last_error()
