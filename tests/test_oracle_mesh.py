"""The static tables (mesh.F) built two independent ways must agree bit for bit.

The library builds FDXE/FDYE/AREAS, NeiTab, CSR_POSITION, the boundary
tables and the cold-start state in csrc/mesh_prep.cpp; the oracle restates
the same reference routines in oracle/oracle_mesh.cpp.  Every parity test
hands the oracle its own tables, so these tests are what ties the two
inputs together.  No GPU is needed.
"""
import ctypes as C
import math

import numpy as np
import pytest


def _cases(orc):
    from adcirc_b200 import model
    yield "channel", model.channel_case
    yield "beach", model.beach_case
    yield "river2", lambda **k: model.channel_case(river=0.5, river_type=2, **k)
    yield "river22", lambda **k: model.channel_case(river=0.5, river_type=22, **k)
    yield "radiation", lambda **k: model.channel_case(radiation=True, **k)
    yield "river52", lambda **k: model.channel_case(river=0.5, river_type=52, flux_settling=0.02, **k)
    yield "zerograd", lambda **k: model.channel_case(zero_gradient=True, **k)
    yield "river32", lambda **k: model.channel_case(river=0.5, river_type=32, **k)
    yield "zerograd41", lambda **k: model.channel_case(zero_gradient=41, **k)
    yield "surge30k", lambda **k: model.surge_case(target_nodes=30_000, **k)
    yield "barrier13", lambda **k: model.channel_case(barrier=-0.5, barrier_type=13, **k)
    yield "levee24", lambda **k: model.channel_case(levee=0.0, levee_type=24, **k)
    yield "pipes5", lambda **k: model.channel_case(levee=1.0, levee_type=5, pipe=(0.0, 1.0, 1.0), **k)
    yield "series", lambda **k: model.channel_case(river=0.5, elev_series=150.0, flux_series=300.0,
                                                   series_hours=1.0, **k)


@pytest.mark.parametrize("name", ["channel", "beach", "river2", "river22", "radiation", "river52",
                                  "zerograd", "river32", "zerograd41", "surge30k", "barrier13",
                                  "levee24", "pipes5", "series"])
def test_case_tables_match(lib, orc, name):
    fn = dict(_cases(orc))[name]
    a = fn()
    b = fn(prep=orc.mesh_prep())
    assert a.sizes == b.sizes
    bad = [k for k in a.arrays if not np.array_equal(a.arrays[k], b.arrays[k])]
    assert not bad, f"tables differ: {bad}"
    # the tables are non-trivial: angle-sorted neighbours and real boundary codes
    assert a.sizes["neimax"] >= 7 and (a.arrays["csr_position"] >= 2).all()


def _boundary(fn, x, y, segs, cos_inner):
    from adcirc_b200._lib import dp_, ip_, ptr
    ibtype = np.array([t for t, _ in segs], np.int32)
    nodes = [np.asarray(s, np.int32) for _, s in segs]
    seg_ptr = np.zeros(len(nodes) + 1, np.int32)
    seg_ptr[1:] = np.cumsum([s.size for s in nodes])
    seg_nodes = np.concatenate(nodes).astype(np.int32)
    nmax = int(seg_nodes.size + len(nodes) + 1)
    nbv, lbc, me2gw = (np.zeros(nmax, np.int32) for _ in range(3))
    csii, siii, blen = (np.zeros(nmax) for _ in range(3))
    nvel, nvelme = C.c_int(0), C.c_int(0)
    rc = fn(x.size, ptr(x, dp_), ptr(y, dp_), len(nodes), ptr(ibtype, ip_), ptr(seg_ptr, ip_),
            ptr(seg_nodes, ip_), cos_inner, nmax, C.byref(nvel), ptr(nbv, ip_), ptr(lbc, ip_),
            ptr(csii, dp_), ptr(siii, dp_), C.byref(nvelme), ptr(me2gw, ip_), ptr(blen, dp_))
    return rc, nvel.value, nvelme.value, nbv, lbc, csii, siii, me2gw, blen


def test_boundary_setup_islands_and_overlaps(lib, orc):
    """Segments the named cases do not have: islands given open (closed
    here), a two-node island (FLG_IBLEN2), a closed external loop, and
    specified-flow segments overlapping no-flow ones at both ends."""
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 1e4, 60)
    y = rng.uniform(0, 1e4, 60)
    segs = [
        (0, [1, 2, 3, 4, 5]),
        (2, [5, 6, 7, 8]),            # flow segment starting on the last no-flow node
        (20, [8, 9, 10, 1]),          # ends on the very first boundary node
        (1, [11, 12, 13, 14]),        # island given open
        (21, [15, 16]),               # two-node island
        (11, [17, 18, 19, 20, 17]),   # island given closed
        (10, [21, 22, 23, 24, 21]),   # closed external loop
        (12, [24, 25, 26]),           # flow segment starting on the loop's node
    ]
    cos_inner = math.cos(math.radians(110.0))
    g = _boundary(lib.adc_boundary_setup, x, y, segs, cos_inner)
    o = _boundary(orc.load().orc_boundary_setup, x, y, segs, cos_inner)
    assert g[0] == 0 and o[0] == 0
    assert g[1:3] == o[1:3]
    for k in range(3, 9):
        assert np.array_equal(g[k], o[k]), k
    assert 10 in g[4] or 11 in g[4] or 12 in g[4]   # some inner angles zero the slip


def test_neighb_rejects_coincident_nodes(orc):
    """NEIGHB stops on coincident nodes (neighb_terminateDuplicateNode)."""
    from adcirc_b200._lib import dp_, ip_, ptr
    x = np.array([0.0, 1.0, 0.0, 0.0])
    y = np.array([0.0, 0.0, 1.0, 0.0])
    nm = np.asfortranarray(np.array([[1, 2, 3], [1, 2, 4]], np.int32))
    nneigh = np.zeros(4, np.int32)
    neitab = np.zeros((4, 6), np.int32, order="F")
    mx = C.c_int(0)
    rc = orc.load().orc_mesh_neighb(4, 2, 6, ptr(x, dp_), ptr(y, dp_), ptr(nm, ip_),
                                    ptr(nneigh, ip_), ptr(neitab, ip_), C.byref(mx))
    assert rc == -4


def test_neitabele_packs_each_ring(lib, orc):
    """NeiTabEle (mesh.F:3248-3283): every interior node lists one element
    per neighbour pair of its ring, every boundary node one fewer, each
    element holding the node."""
    from adcirc_b200 import model
    c = model.channel_case(prep=orc.mesh_prep())
    a = c.arrays
    te, nn, nm = a["neitabele"], a["nneigh"], a["nm"] - 1
    nv = c.sizes["nvel"]
    boundary = np.zeros(c.sizes["np"], bool)
    boundary[a["nbv"][:nv] - 1] = True
    boundary[a["nbd"] - 1] = True
    cnt = (te > 0).sum(axis=1)
    assert np.array_equal(cnt[~boundary], nn[~boundary] - 1)
    assert np.array_equal(cnt[boundary], nn[boundary] - 2)
    for i in range(0, c.sizes["np"], 97):
        for e in te[i][te[i] > 0] - 1:
            assert i in nm[e]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_meshes_tables_match(lib, orc, seed):
    """Scattered-point Delaunay meshes (half the elements listed clockwise,
    irregular valence, an open segment and a land segment around the hull):
    the library's and the oracle's table builders agree bit for bit."""
    from scipy.spatial import Delaunay
    from adcirc_b200 import model
    from adcirc_b200.meshgen import RawMesh
    rng = np.random.default_rng(seed)
    n = 400
    pts = rng.uniform(0.0, 1.0e4, size=(n, 2))
    tri = Delaunay(pts)
    nm = tri.simplices.astype(np.int64)
    flip = rng.random(nm.shape[0]) < 0.5            # half the elements clockwise
    nm[flip] = nm[flip][:, [0, 2, 1]]
    hull = tri.convex_hull                           # edges of the outer boundary
    # walk the hull as one ordered loop
    nxt = {}
    for a_, b_ in hull:
        nxt.setdefault(a_, []).append(b_)
        nxt.setdefault(b_, []).append(a_)
    loop = [hull[0][0]]
    prev = None
    while True:
        cur = loop[-1]
        cand = [v for v in nxt[cur] if v != prev]
        prev, nx_ = cur, cand[0]
        if nx_ == loop[0]:
            break
        loop.append(nx_)
    loop = np.asarray(loop, np.int64)
    open_nodes = loop[:6]
    land = loop[5:]
    raw = RawMesh(f"random{seed}", pts[:, 0].copy(), pts[:, 1].copy(),
                  rng.uniform(2.0, 10.0, n), nm, open_nodes, [(0, land)], {"lx": 1e4, "ly": 1e4})
    sched = model.Schedule(dt=2.0)
    tides = [(1.4e-4, 0.0, 1.0, np.full(open_nodes.size, 0.3), np.zeros(open_nodes.size))]
    a = model.build_case(raw, model.default_params(2.0), sched, tides)
    b = model.build_case(raw, model.default_params(2.0), sched, tides, prep=orc.mesh_prep())
    assert a.sizes == b.sizes
    bad = [k for k in a.arrays if not np.array_equal(a.arrays[k], b.arrays[k])]
    assert not bad, f"tables differ: {bad}"
