"""The reference's binary hotstart file (fort.67/68): the record layout of
writeHotstart (write_output.F:4900-5154) and what hstart.F (:500-560,
764-768, 857-883) derives from it.  Host code only; the oracle steps the
runs."""
import struct

import numpy as np
import pytest

from adcirc_b200 import adcirc_io, model


def _stepped(orc, n, **kw):
    case = model.channel_case(**kw)
    om = orc.OracleModel(case)
    om.run(1, n)
    return case, om


def test_fort67_layout_and_round_trip(lib, orc, tmp_path):
    case, om = _stepped(orc, 30)
    om.close()
    p = tmp_path / "fort.67"
    adcirc_io.write_fort67(p, case, 30, 150.0)
    raw = p.read_bytes()
    npn, ne = case.sizes["np"], case.sizes["ne"]
    assert len(raw) == 8 * (8 + 5 * npn + npn + ne + 8 * npn + 18)
    rec = lambda r: raw[8 * r:8 * r + 8]
    assert struct.unpack("<i", rec(0)[:4])[0] == (1 << 20) | (2 << 10)   # FileFmtVersion 1.2.0
    assert struct.unpack("<d", rec(2))[0] == 150.0                        # TimeLoc
    assert [struct.unpack("<i", rec(r)[:4])[0] for r in (3, 4, 5, 6, 7)] == [30, npn, ne, npn, ne]
    assert struct.unpack("<d", rec(8 + npn + 3))[0] == case.arrays["eta2"][3]   # ETA2(4)
    back = adcirc_io.read_fort67(p)
    assert back["it"] == 30 and back["timeloc"] == 150.0 and back["im"] == 0
    for k in ("eta1", "eta2", "uu2", "vv2", "nodecode", "noff"):
        assert np.array_equal(back[k], case.arrays[k]), k


def test_fort67_refuses_other_versions_and_meshes(lib, orc, tmp_path):
    case, om = _stepped(orc, 2)
    om.close()
    p = tmp_path / "fort.67"
    adcirc_io.write_fort67(p, case, 2, 10.0)
    raw = bytearray(p.read_bytes())
    raw[0:4] = struct.pack("<i", (1 << 20) | (3 << 10))
    q = tmp_path / "v13.67"
    q.write_bytes(bytes(raw))
    with pytest.raises(OSError, match="version 1.3"):
        adcirc_io.read_fort67(q)
    beach = model.beach_case()
    with pytest.raises(ValueError, match="another mesh"):
        model.apply_hotstart(beach, adcirc_io.read_fort67(p))


def test_run_continues_from_a_reference_hotstart(lib, orc, tmp_path):
    """A run stopped at step 60 and written as fort.67, then a fresh case
    loaded from it as hstart.F loads it, continues alongside the
    uninterrupted run: the reference's hotstart carries only the primary
    state, so the two agree to the JCG tolerance, not bit for bit."""
    full, om = _stepped(orc, 60)
    p = tmp_path / "fort.67"
    adcirc_io.write_fort67(p, full, 60, full.schedule.step(60).timeloc)
    om.run(61, 40)
    om.close()
    seeded = model.channel_case()
    iths = model.apply_hotstart(seeded, adcirc_io.read_fort67(p))
    assert iths == 60
    storm = model.channel_case(vortex=True)
    model.apply_hotstart(storm, adcirc_io.read_fort67(p))
    assert storm.vortex.start_time == 300.0   # NWS08INIT picks the fix pair from TimeLoc
    assert np.array_equal(seeded.arrays["qx2"], seeded.arrays["uu2"] * seeded.arrays["h2"])
    om2 = orc.OracleModel(seeded)
    om2.run(iths + 1, 40)
    om2.close()
    d = np.abs(seeded.arrays["eta2"] - full.arrays["eta2"]).max()
    assert d < 1e-7 * np.abs(full.arrays["eta2"]).max()
    assert np.array_equal(seeded.arrays["nodecode"], full.arrays["nodecode"])


def test_series_positioned_at_the_hotstart(lib, orc):
    """hstart.F:857-883 replays the fort.19 read-ahead up to ITHS: the
    seeded series holds the same record pair and times as the run that
    got there step by step."""
    case = model.channel_case(elev_series=150.0, series_hours=1.0)
    s = case.elev_series
    sched = case.schedule
    for iths in (1, 29, 30, 31, 95, 300):
        t = model.series_at_hotstart(s, iths, sched.step(iths).timeloc, sched)
        # the run's own pair after step iths (the read-ahead of every step)
        t1, t2, k = s.start_time, s.start_time + s.interval, 0
        for it in range(1, iths + 1):
            if sched.step(it).timeloc > t2:
                t1, t2, k = t2, t2 + s.interval, k + 1
        assert t.start_time == t1 and np.array_equal(t.values, s.values[k:]), iths
