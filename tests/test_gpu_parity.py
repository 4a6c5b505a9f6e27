"""GPU parity: libadcgpu (CUDA, sm_100a) against the CPU oracle.

Tolerances (FP64 path): eta, velocity and flux fields within 1e-9 relative
to the field's maximum magnitude; JCG iteration counts and the integer
wet/dry flags (NODECODE, NOFF) exact.  The only arithmetic allowed to
differ is the order of the JCG dot-product sums (tree vs sequential) and
CUDA's cos at elevation-boundary nodes, both at the 1e-16 level.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9
FIELDS = ("eta1", "eta2", "etas", "uu2", "vv2", "qx2", "qy2", "h2", "tk", "totalarea")


def _rel(a, b):
    scale = max(np.abs(b).max(), 1e-30)
    return float(np.abs(a - b).max() / scale)


def oracle_and_gpu_cases(case_fn):
    """(oracle case, GPU case): the oracle's built with its own restatement of
    the static tables (oracle/oracle_mesh.cpp), the GPU's with the library's;
    the two sets must agree bit for bit before any step is compared."""
    import oracle
    c0 = case_fn(prep=oracle.mesh_prep())
    cg = case_fn()
    assert c0.sizes == cg.sizes
    bad = [k for k in c0.arrays if not np.array_equal(c0.arrays[k], cg.arrays[k])]
    assert not bad, f"static tables differ: {bad}"
    return c0, cg


def _pair(case_fn, nsteps, use_run=False):
    """`case_fn(prep=...)` builds the case; see oracle_and_gpu_cases."""
    import oracle
    from adcirc_b200 import model
    c0, cg = oracle_and_gpu_cases(case_fn)
    orc = oracle.OracleModel(c0)
    gpu = model.GpuModel(cg)
    its_o = np.array([orc.step(it).numitr for it in range(1, nsteps + 1)])
    if use_run:
        its_g, _ = gpu.run(1, nsteps)
    else:
        its_g = np.array([gpu.step(it).numitr for it in range(1, nsteps + 1)])
    gpu.sync_to_host()
    gpu.close()
    orc.close()
    return c0, cg, its_o, np.asarray(its_g)


def _check(c0, cg, its_o, its_g):
    a, b = c0.arrays, cg.arrays
    errs = {f: _rel(b[f], a[f]) for f in FIELDS}
    bad = {f: e for f, e in errs.items() if not e <= REL_TOL}
    assert not bad, f"fields beyond {REL_TOL}: {bad}"
    # COEF as the host sees it after sync: rebuilt, scaled and unscaled by
    # every solve, including the drift a solve leaves for the next step
    # (only EP at elevation-boundary rows comes from a differently ordered sum)
    errs["coef"] = _rel(b["coef"], a["coef"])
    assert errs["coef"] <= 1e-12, f"COEF differs: {errs['coef']}"
    assert np.array_equal(a["nodecode"], b["nodecode"])
    assert np.array_equal(a["noff"], b["noff"])
    mism = int(np.sum(its_o != its_g))
    assert mism == 0, f"JCG iteration counts differ in {mism} steps: {its_o} vs {its_g}"
    return errs


def test_channel_steps(lib, orc):
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(model.channel_case, 60)
    _check(c0, cg, io, ig)
    assert io.min() > 0


def test_channel_graph_run(lib, orc):
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(model.channel_case, 120, use_run=True)
    _check(c0, cg, io, ig)


def test_beach_wetdry(lib, orc):
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(model.beach_case, 400, use_run=True)
    errs = _check(c0, cg, io, ig)
    a = c0.arrays
    # the case must actually exercise drying
    assert (a["nodecode"] == 0).sum() > 0 and (a["nodecode"] == 1).sum() > 0
    assert errs["eta2"] <= REL_TOL


def test_lake_at_rest(lib):
    from adcirc_b200 import model
    case = model.channel_case(amp=0.0)
    gpu = model.GpuModel(case)
    numitr, last = gpu.run(1, 50)
    gpu.sync_to_host()
    a = case.arrays
    assert np.all(a["eta2"] == 0.0) and np.all(a["uu2"] == 0.0) and np.all(a["vv2"] == 0.0)
    assert np.all(numitr == 0)


def test_deterministic(lib):
    from adcirc_b200 import model
    outs = []
    for _ in range(2):
        case = model.beach_case()
        gpu = model.GpuModel(case)
        gpu.run(1, 200)
        gpu.sync_to_host()
        outs.append((case.arrays["eta2"].copy(), case.arrays["uu2"].copy()))
        gpu.close()
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def _jcg_system(orc_mod):
    """A GWCE system (COEF, NeiTab, GWCE_LV, ETAS) from the channel case."""
    from adcirc_b200 import model
    case = model.channel_case()
    om = orc_mod.OracleModel(case)
    for it in range(1, 4):
        om.step(it)
    om.shift_friction(4)
    om.close()
    a = case.arrays
    n = case.sizes["np"]
    rng = np.random.default_rng(7)
    return (n, case.sizes["mnei"], a["neitab"].copy(order="F"), a["coef"].copy(order="F"),
            rng.standard_normal(n), 1e-3 * rng.standard_normal(n))


def _call_adc_jcg(lib, n, mnei, jcoef, coef, rhs, u, iparm, rparm):
    from adcirc_b200._lib import dp_, ip_, ptr
    nw = 4 * n + 4 * int(iparm[0])
    wksp = np.zeros(nw)
    iwksp = np.zeros(3 * n, np.int32)
    ier = C.c_int(0)
    lib.adc_jcg(C.byref(C.c_int(n)), C.byref(C.c_int(n)), C.byref(C.c_int(mnei)), ptr(jcoef, ip_),
                ptr(coef, dp_), ptr(rhs, dp_), ptr(u, dp_), ptr(iwksp, ip_), C.byref(C.c_int(nw)),
                ptr(wksp, dp_), ptr(iparm, ip_), ptr(rparm, dp_), C.byref(ier))
    return ier.value


@pytest.mark.parametrize("itmax,tol", [(200, 1e-10), (3, 1e-10)])
def test_jcg_dropin(lib, orc, itmax, tol):
    n, mnei, jc, cf, rhs, u0 = _jcg_system(orc)
    res = []
    lib.adc_jcg_reset()
    orc.load().orc_itpack_reset()
    for impl in ("gpu", "orc"):
        jcoef, coef, r, u = jc.copy(order="F"), cf.copy(order="F"), rhs.copy(), u0.copy()
        iparm, rparm = orc.dfault()
        iparm[0] = itmax
        rparm[0] = tol
        if impl == "gpu":
            ier = _call_adc_jcg(lib, n, mnei, jcoef, coef, r, u, iparm, rparm)
        else:
            ier = orc.jcg(n, n, mnei, jcoef, coef, r, u, iparm, rparm)
        res.append((ier, u, coef, jcoef, r, iparm.copy(), rparm.copy()))
    g, o = res
    assert g[0] == o[0]
    assert g[5][0] == o[5][0], "iteration count"
    assert _rel(g[1], o[1]) <= 1e-9
    assert np.array_equal(g[3], o[3])
    assert _rel(g[2], o[2]) <= 1e-13      # the scal/unscal drift of COEF
    assert _rel(g[4], o[4]) <= 1e-13      # rhs restored
    if itmax == 3:
        assert o[0] == 13 and abs(g[6][0] - o[6][0]) <= 1e-9 * abs(o[6][0])


@pytest.mark.parametrize("ny", [401, 2101])
def test_w1_chain_burst(lib, orc, ny):
    """A wetting front across a long beach: one wet/dry pass with hundreds
    (ny=401) to thousands (ny=2101) of W1 events whose TK updates chain
    through shared nodes from row to row.  The order-dependent result
    (wetdry.F:593-618) must match the sequential oracle bit for bit, for the
    block-wide resolution of short lists and the batched one of long lists."""
    import oracle
    from adcirc_b200 import _lib, meshgen, model
    raw = meshgen.channel_mesh(nx=41, ny=ny, lx=4e3, ly=0.1e3 * (ny - 1), depth0=3.0, depth1=-1.5)
    rng = np.random.default_rng(7)
    eta0 = np.where(raw.dp > 0.05, rng.uniform(0.5, 1.0, raw.dp.size), 0.0)
    params = model.default_params(0.1)
    tides = [(1e-4, 0.0, 1.0, np.zeros(raw.open_nodes.size), np.zeros(raw.open_nodes.size))]
    tk = rng.uniform(0.0, 8.0, raw.dp.size)

    def build(**k):
        c = model.build_case(raw, params, model.Schedule(dt=0.1, nramp=0), tides, eta0=eta0, **k)
        c.arrays["tk"][:] = tk
        c.arrays["tkm"][:] = 0.0
        c.arrays["tkm"][0::3] = tk
        c.arrays["tkm"][1::3] = tk
        return c
    c0, cg = oracle_and_gpu_cases(build)
    base = cg
    o = oracle.OracleModel(c0)
    oo = o.wetdry(1)
    g = model.GpuModel(cg)
    go = _lib.AdcStepOut()
    assert lib.adc_wetdry(g.h, C.byref(base.schedule.step(1)), C.byref(go)) == 0
    g.sync_to_host()
    g.close()
    o.close()
    assert go.n_w1_events == oo.n_w1_events
    assert (300 if ny == 401 else 2000) <= go.n_w1_events, go.n_w1_events
    for f in ("tk", "tkm", "nodecode", "nnodecode", "noff", "eta2"):
        assert np.array_equal(cg.arrays[f], c0.arrays[f]), f


@pytest.mark.parametrize("river_type", [2, 22])
def test_channel_river_flux(lib, orc, river_type):
    """A specified-flux (river) boundary at the closed end: the periodic flux
    forcing, the GWCE boundary integral (gwce.F:1737-1834) and, for IBTYPE 2,
    the specified normal velocity of the momentum equation, against the
    oracle over a graph-replayed run."""
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(river=0.5, river_type=river_type, **k), 150,
                           use_run=True)
    _check(c0, cg, io, ig)
    a = c0.arrays
    east = a["x"] > 59.9e3
    assert a["uu2"][east].mean() < -0.02   # the inflow reaches the boundary nodes


def test_channel_radiation_boundary(lib, orc):
    """A radiation boundary (IBTYPE 30) at the channel's east end: the
    discharge of the latest velocity (timestep.F:932-940) and the radiation
    force -sqrt(g H1) ETAS / DT - TAU0 QN1 of the GWCE boundary integral
    (gwce.F:1783-1790), against the oracle over a graph-replayed run long
    enough for the tide to reach and leave through the boundary."""
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(radiation=True, **k), 1500, use_run=True)
    _check(c0, cg, io, ig)
    a = c0.arrays
    east = a["x"] > 59.9e3
    assert a["uu2"][east].mean() > 0.02   # the tide leaves through the boundary


def test_channel_river_radiation(lib, orc):
    """A river-radiation boundary (IBTYPE 52) with a flux settling time: the
    tide waits for the river flux to settle (NRAMP 2, timestep.F:314-345),
    the discharge elevation is taken at FluxSettlingIT (timestep.F:906-926)
    and the radiation term joins the specified flux after it (gwce.F:
    1805-1815), against the oracle over a graph-replayed run."""
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(river=0.5, river_type=52, flux_settling=0.02,
                                                          **k), 800, use_run=True)
    _check(c0, cg, io, ig)
    a = c0.arrays
    east = a["x"] > 59.9e3
    assert a["uu2"][east].mean() < -0.02   # the river enters


def test_channel_zero_gradient_boundary(lib, orc):
    """A zero-normal-velocity-gradient boundary (IBTYPE 40) at the east end:
    the discharge of the latest velocity (timestep.F:945-952), its force in
    the GWCE boundary integral (gwce.F:1804-1805) and the interpolated
    boundary velocity of the momentum step (momentum.F:1157-1174), against
    the oracle over a graph-replayed run."""
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(zero_gradient=True, **k), 1500, use_run=True)
    _check(c0, cg, io, ig)
    a = c0.arrays
    east = a["x"] > 59.9e3
    assert a["uu2"][east].mean() > 0.02


def test_channel_coupled_flux_radiation(lib, orc):
    """A coupled flux/radiation boundary (IBTYPE 32): flux and elevation
    constituents (timestep.F:861-880) and the radiation condition against
    the specified elevation in the GWCE boundary integral (gwce.F:
    1792-1797), against the oracle over a graph-replayed run."""
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(river=0.5, river_type=32, **k), 1000,
                           use_run=True)
    _check(c0, cg, io, ig)
    a = c0.arrays
    east = a["x"] > 59.9e3
    assert a["uu2"][east].mean() < -0.02


def test_channel_galerkin_zero_gradient_boundary(lib, orc):
    """The Galerkin zero-normal-velocity-gradient boundary (IBTYPE 41): the
    momentum equations of its nodes replaced by the normal derivative over
    the ring's elements (momentum.F:864-933, NeiTabEle used positionally as
    there), against the oracle over a graph-replayed run."""
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(zero_gradient=41, **k), 1500, use_run=True)
    _check(c0, cg, io, ig)
    a = c0.arrays
    east = a["x"] > 59.9e3
    assert a["uu2"][east].mean() > 0.02


def test_channel_elevation_series(lib, orc):
    """A non-periodic elevation boundary (fort.19, NBFR 0): the record pair
    the run holds moves on as TimeLoc passes each record time and the
    boundary elevation is their interpolation (gwce.F:1659-1674), against
    the oracle over a graph-replayed run through twenty record changes."""
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(elev_series=150.0, series_hours=1.0, **k),
                           600, use_run=True)
    _check(c0, cg, io, ig)


@pytest.mark.parametrize("river_type", [2, 32])
def test_channel_flux_series(lib, orc, river_type):
    """A river boundary driven by a fort.20 series (NFFR 0): QN2 (and EN2 at
    IBTYPE 32) interpolated between the records the run holds (timestep.F:
    882-903), against the oracle over a graph-replayed run."""
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(river=0.5, river_type=river_type,
                                                          flux_series=300.0, series_hours=1.0, **k),
                           600, use_run=True)
    _check(c0, cg, io, ig)
    a = c0.arrays
    east = a["x"] > 59.9e3
    assert a["uu2"][east].mean() < -0.02


@pytest.mark.parametrize("btype,crest,nsteps", [(3, -0.05, 1500), (13, -0.5, 400), (23, -0.5, 400)])
def test_channel_external_barrier(lib, orc, btype, crest, nsteps):
    """An external barrier (IBTYPE 3/13/23) at the east end: the weir outflow
    over the crest as QN2 (weir_boundary.F90:1727-1763), its GWCE boundary
    integral and, for 3 and 13, the normal velocity of the momentum step,
    against the oracle over a graph-replayed run.  With the crest at -0.05 m
    the run passes from no outflow to outflow when the tide arrives."""
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(barrier=crest, barrier_type=btype, **k),
                           nsteps, use_run=True)
    _check(c0, cg, io, ig)
    a = c0.arrays
    east = a["x"] > 59.9e3
    assert a["uu2"][east].mean() > 0.001   # water leaves over the barrier


@pytest.mark.parametrize("ltype", [4, 24])
def test_channel_internal_barrier(lib, orc, ltype):
    """An internal barrier (IBTYPE 4/24) between the tidal channel and a dry
    polder: the paired flow over the crest (weir_boundary.F90:1775-1942,
    the wet-edge rules included), the receiving-node flags and the polder's
    wetting through NIBCNT (wetdry.F:813-816, 1086-1090, 1114), against the
    oracle over a graph-replayed run."""
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(levee=0.0, levee_type=ltype, amp=2.0, **k),
                           1000, use_run=True)
    _check(c0, cg, io, ig)
    a = c0.arrays
    east = a["x"] > 30.0e3 + 1.0
    assert a["nodecode"][east].sum() > 100   # the polder has begun to flood


@pytest.mark.parametrize("ltype", [5, 25])
def test_channel_barrier_pipes(lib, orc, ltype):
    """A barrier too high to overtop with a pipe under every pair (IBTYPE
    5/25): the pipe discharge added to the barrier flux (weir_boundary.F90:
    2469-2579, timestep.F:1034-1044) floods the polder, against the oracle
    over a graph-replayed run."""
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(levee=10.0, levee_type=ltype,
                                                          pipe=(-0.5, 1.0, 1.0), amp=2.0, **k),
                           1000, use_run=True)
    _check(c0, cg, io, ig)
    a = c0.arrays
    assert a["nodecode"][a["x"] > 30.0e3 + 1.0].sum() > 100
