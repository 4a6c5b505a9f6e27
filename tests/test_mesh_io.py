"""fort.14 and fort.63/64 host I/O (no GPU): round trips, the reference's
read14 conventions (arbitrary node labels, D exponents, trailing columns)
and the Fortran formats of the output files."""
import numpy as np
import pytest


def test_fort14_round_trip(lib, tmp_path):
    from adcirc_b200 import adcirc_io, meshgen
    raw = meshgen.beach_mesh()
    p = tmp_path / "fort.14"
    adcirc_io.write_fort14(raw, p, title="beach")
    back = adcirc_io.read_fort14(p)
    assert back.name == "beach"
    for f in ("x", "y", "dp"):
        assert np.array_equal(getattr(back, f), getattr(raw, f)), f   # 17 digits round-trip
    assert np.array_equal(back.nm, raw.nm)
    assert np.array_equal(back.open_nodes, raw.open_nodes)
    assert len(back.land_segments) == len(raw.land_segments)
    for (t0, s0), (t1, s1) in zip(raw.land_segments, back.land_segments):
        assert t0 == t1 and np.array_equal(np.asarray(s0), s1)


def test_fort14_case_runs_like_original(lib, tmp_path):
    """A mesh read back from fort.14 builds the same bound arrays."""
    from adcirc_b200 import adcirc_io, meshgen, model
    raw = meshgen.beach_mesh()
    p = tmp_path / "fort.14"
    adcirc_io.write_fort14(raw, p)
    raw2 = adcirc_io.read_fort14(p)
    raw2.meta.update(raw.meta)
    sched = model.Schedule(dt=2.0, nramp=0)
    tides = [(1e-4, 0.0, 1.0, np.full(raw.open_nodes.size, 0.5), np.zeros(raw.open_nodes.size))]
    a = model.build_case(raw, model.default_params(2.0), sched, tides).arrays
    b = model.build_case(raw2, model.default_params(2.0), sched, tides).arrays
    for k in ("neitab", "nneigh", "csr_position", "fdxe", "fdye", "areas", "nbv", "lbcodei", "csii",
              "siii", "nodecode", "totalarea"):
        assert np.array_equal(a[k], b[k]), k


def test_fort14_labels_and_fortran_numbers(lib, tmp_path):
    from adcirc_b200 import adcirc_io
    text = """quad with odd labels
2 4
10 0.0 0.0 1.5D0
20 1.0D3 0.0 2.0
30 1000.0, 1000.0, 2.5
40 0.0 1.0E+03 3.0
1 3 10 20 30
2 3 10 30 40
1 ! NOPE
2 ! NETA
2 0
10
40
1
3
3 0
20
30
40
"""
    p = tmp_path / "fort.14"
    p.write_text(text)
    m = adcirc_io.read_fort14(p)
    assert m.name == "quad with odd labels"
    assert np.array_equal(m.x, [0.0, 1000.0, 1000.0, 0.0]) and np.array_equal(m.dp, [1.5, 2.0, 2.5, 3.0])
    assert np.array_equal(m.nm, [[0, 1, 2], [0, 2, 3]])
    assert np.array_equal(m.open_nodes, [0, 3])
    assert m.land_segments[0][0] == 0 and np.array_equal(m.land_segments[0][1], [1, 2, 3])


def test_fort14_periodic_unsupported(lib, tmp_path):
    """Periodic boundary segments (IBTYPE 94) are refused."""
    from adcirc_b200 import _lib, adcirc_io
    text = "t\n1 3\n1 0 0 1\n2 1 0 1\n3 0 1 1\n1 3 1 2 3\n0\n0\n1\n2\n2 94\n1 2\n3 1\n"
    p = tmp_path / "fort.14"
    p.write_text(text)
    dims = np.zeros(6, np.int32)
    rc = lib.adc_fort14_dims(str(p).encode(), dims.ctypes.data_as(_lib.ip_))
    assert rc == _lib.ADC_ERR_UNSUPPORTED
    with pytest.raises(OSError):
        adcirc_io.read_fort14(p)


def test_fort14_external_barrier(lib, tmp_path):
    """IBTYPE 3/13/23 node lines carry BARLANHT and BARLANCFSP (read14,
    mesh.F:460-473); they survive a write and a read."""
    from adcirc_b200 import adcirc_io
    text = ("t\n1 3\n1 0 0 1\n2 1 0 1\n3 0 1 1\n1 3 1 2 3\n0\n0\n2\n5\n"
            "2 3\n1 0.5 1.0\n2 0.6D0 0.9\n3 0\n2\n3\n1\n")
    p = tmp_path / "fort.14"
    p.write_text(text)
    m = adcirc_io.read_fort14(p)
    assert [t for t, _ in m.land_segments] == [3, 0]
    assert np.array_equal(m.barriers[0][0], [0.5, 0.6]) and np.array_equal(m.barriers[0][1], [1.0, 0.9])
    assert 1 not in m.barriers
    q = tmp_path / "back.14"
    adcirc_io.write_fort14(m, q)
    m2 = adcirc_io.read_fort14(q)
    assert np.array_equal(m2.barriers[0][0], m.barriers[0][0])
    assert np.array_equal(m2.barriers[0][1], m.barriers[0][1])
    bad = tmp_path / "bad.14"
    bad.write_text(text.replace("2 0.6D0 0.9", "2"))
    with pytest.raises(OSError, match="external barrier"):
        adcirc_io.read_fort14(bad)


def test_fort14_internal_barrier(lib, tmp_path):
    """IBTYPE 4/24 node lines hold the pair, the crest and both discharge
    coefficients (read14, mesh.F:479-495); the pairs count twice in NVEL,
    and a mesh written and read back builds the same bound arrays."""
    from adcirc_b200 import adcirc_io, meshgen, model
    raw = meshgen.levee_channel_mesh(0.25, 24, cfsb=0.9, cfsp=0.8)
    p = tmp_path / "fort.14"
    adcirc_io.write_fort14(raw, p)
    text = p.read_text().splitlines()
    nbou_line = len(text) - 2 - sum(len(s) + 1 for _, s in raw.land_segments)
    assert int(text[nbou_line].split()[0]) == 2                   # NBOU
    assert int(text[nbou_line + 1].split()[0]) == 281 + 2 * 39   # NVEL
    back = adcirc_io.read_fort14(p)
    assert [t for t, _ in back.land_segments] == [0, 24]
    b0, b1 = raw.barriers[1], back.barriers[1]
    for u, v in zip(b0, b1):
        assert np.array_equal(np.asarray(u), np.asarray(v))
    sched = model.Schedule(dt=5.0)
    tides = [(1e-4, 0.0, 1.0, np.full(raw.open_nodes.size, 0.5), np.zeros(raw.open_nodes.size))]
    a = model.build_case(raw, model.default_params(5.0), sched, tides).arrays
    b = model.build_case(back, model.default_params(5.0), sched, tides).arrays
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(a["nvell"], [281, 39])
    lbc = a["lbcodei"]
    assert (lbc == 24).sum() == 78
    # front face pairs with the back face, the back face runs backwards
    front = np.nonzero(lbc == 24)[0][:39]
    assert np.array_equal(a["ibconn"][front] - 1, b1[3])
    assert np.array_equal(a["nbv"][front[-1] + 1:front[-1] + 40] - 1, b1[3][::-1])


def test_fort14_barrier_pipes(lib, tmp_path):
    """IBTYPE 5/25 pairs also carry the pipe's crown height, coefficient and
    diameter (mesh.F:506-524); they survive the file and reach the bound
    arrays in face order."""
    from adcirc_b200 import adcirc_io, meshgen, model
    raw = meshgen.levee_channel_mesh(2.0, 25, pipe=(0.3, 1.5, 0.8))
    p = tmp_path / "fort.14"
    adcirc_io.write_fort14(raw, p)
    back = adcirc_io.read_fort14(p)
    assert [t for t, _ in back.land_segments] == [0, 25]
    for u, v in zip(raw.barriers[1], back.barriers[1]):
        assert np.array_equal(np.asarray(u), np.asarray(v))
    sched = model.Schedule(dt=5.0)
    tides = [(1e-4, 0.0, 1.0, np.full(raw.open_nodes.size, 0.5), np.zeros(raw.open_nodes.size))]
    a = model.build_case(back, model.default_params(5.0), sched, tides).arrays
    on = a["lbcodei"] == 25
    assert on.sum() == 78
    assert np.all(a["pipeht"][on] == 0.3) and np.all(a["pipecoef"][on] == 1.5)
    assert np.all(a["pipediam"][on] == 0.8) and not np.any(a["pipediam"][~on])


def test_fort63_64_format(lib, tmp_path):
    from adcirc_b200 import adcirc_io
    p = tmp_path / "fort.63"
    w = adcirc_io.Fort6x(p, 3, 1, dt_out=60.0, nspool=60, ndsets=2, rundes="surge", runid="r1",
                         agrid="grid")
    eta = np.array([0.125, -1.5e-7, 2.0])
    w.append(3600.0, 3600, eta, nodecode=np.array([1, 1, 0]))
    w.append(7200.0, 7200, eta)
    lines = p.read_text().splitlines()
    # (1X,A32,2X,A24,2X,A24)
    assert lines[0] == " " + "surge".ljust(32) + "  " + "r1".ljust(24) + "  " + "grid".ljust(24)
    # (1X,I10,1X,I10,1X,E15.7E3,1X,I8,1X,I5,1X,'FileFmtVersion: ',I10)
    assert lines[1] == " " + "2".rjust(10) + " " + "3".rjust(10) + " " + "0.6000000E+002".rjust(15) + \
        " " + "60".rjust(8) + " " + "1".rjust(5) + " FileFmtVersion: " + str((1 << 20) | (2 << 10)).rjust(10)
    # (2x,1pE20.10E3,5X,I10)
    assert lines[2] == "  " + "3.6000000000E+003".rjust(20) + "     " + "3600".rjust(10)
    # (2x, i8, 2x, 1pE20.10E3)
    assert lines[3] == "  " + "1".rjust(8) + "  " + "1.2500000000E-001".rjust(20)
    assert lines[4] == "  " + "2".rjust(8) + "  " + "-1.5000000000E-007".rjust(20)
    assert lines[5] == "  " + "3".rjust(8) + "  " + "-9.9999000000E+004".rjust(20)   # dry
    assert float(lines[9].split()[1]) == 2.0
    q = tmp_path / "fort.64"
    w2 = adcirc_io.Fort6x(q, 2, 2, dt_out=1.0, nspool=1, ndsets=1)
    w2.append(1.0, 1, np.array([0.5, 0.25]), np.array([-0.5, 1e-300]))
    l2 = q.read_text().splitlines()
    assert l2[3] == "  " + "1".rjust(8) + "  " + "5.0000000000E-001".rjust(20) + "-5.0000000000E-001".rjust(20)
    assert l2[4].endswith("1.0000000000E-300")
