"""Known answers the oracle must meet (no GPU): volume conservation in a
closed basin, the inflow mass balance, and mirror symmetry.  See
kat_cases.py for why each holds for the discrete scheme."""
import numpy as np

import kat_cases as K


def test_closed_basin_conserves_volume(orc):
    c = K.closed_basin(prep=orc.mesh_prep())
    v0 = K.basin_volume(c)
    om = orc.OracleModel(c)
    drift = []
    for it in range(1, 401):
        om.step(it)
        drift.append(K.basin_volume(c) - v0)
    om.close()
    assert np.abs(c.arrays["eta2"]).max() > 0.05          # the hump is still moving
    assert max(abs(d) for d in drift) <= 1e-8 * v0, max(abs(d) for d in drift) / v0


def test_river_inflow_mass_balance(orc):
    c = K.river_basin(prep=orc.mesh_prep())
    om = orc.OracleModel(c)
    om.run(1, 719)
    v1 = K.basin_volume(c)
    om.run(720, 721)
    v2 = K.basin_volume(c)
    om.close()
    q = K.inflow_volume(c, 720, 1441)
    assert abs((v2 - v1) - q) <= 1e-6 * q, ((v2 - v1) - q) / q


def test_mirror_symmetry(orc):
    c = K.mirror_channel(prep=orc.mesh_prep())
    om = orc.OracleModel(c)
    om.run(1, 720)
    om.close()
    asym = K.asymmetry(c)
    assert asym["eta"] <= 1e-12 and asym["u"] <= 1e-12 and asym["v"] <= 1e-9, asym


def test_radiation_boundary_passes_the_wave(orc):
    """A radiation boundary (IBTYPE 30) lets the incoming tide leave: at the
    boundary the normal velocity follows the outgoing long-wave relation
    u = eta sqrt(g / H) (the condition gwce.F:1783-1790 imposes), where a
    closed end holds u = 0 and reflects."""
    from adcirc_b200 import model
    c = model.channel_case(radiation=True, prep=orc.mesh_prep())
    om = orc.OracleModel(c)
    om.run(1, 1500)
    om.close()
    a = c.arrays
    east = a["x"] > 59.9e3
    u, eta, h = a["uu2"][east].mean(), a["eta2"][east].mean(), a["h2"][east].mean()
    assert u > 0.02 and eta > 0.02
    ratio = u / (eta * np.sqrt(c.params["g"] / h))
    assert 0.9 <= ratio <= 1.1, ratio


def test_quarter_annulus_matches_the_analytic_tide(orc):
    """Lynch and Gray's quarter-annular harbour (the reference test suite's
    2D case): depth ~ r^2, linear friction, M2 on the outer arc.  The
    oracle's periodic tide matches the closed-form solution (amplitude
    0.30-0.57 m, phase 0-36 degrees) and the error falls with refinement."""
    from adcirc_b200 import model
    errs = []
    for nr, nth in ((11, 16), (21, 31)):
        c = model.quarter_annulus_case(nr=nr, nth=nth, prep=orc.mesh_prep())
        om = orc.OracleModel(c)
        amp, ph = K.harmonic_m2(lambda it, n: om.run(it, n), c)
        om.close()
        errs.append(K.annulus_errors(c, amp, ph))
    (a0, p0), (a1, p1) = errs
    assert a1 <= 5e-3 and p1 <= 0.5, errs
    assert a1 < a0 and p1 < p0, errs


def test_river_radiation_settles_and_holds_the_discharge_level(orc):
    """River radiation (IBTYPE 52): before FluxSettlingIT only the river
    flux drives the channel (the tide is held at zero), the discharge
    elevation is then fixed, and afterwards the boundary keeps carrying the
    river inflow while the tide comes in."""
    from adcirc_b200 import model
    c = model.channel_case(river=0.5, river_type=52, flux_settling=0.02, prep=orc.mesh_prep())
    fsit = c.flux.flux_settling_it
    a = c.arrays
    open_nodes = a["nbd"] - 1
    om = orc.OracleModel(c)
    om.run(1, fsit)
    assert np.abs(a["eta2"][open_nodes]).max() == 0.0     # no tide while settling
    east = a["x"] > 59.9e3
    assert a["uu2"][east].mean() < -0.02                  # the river flows in
    om.run(fsit + 1, 800)
    om.close()
    assert np.abs(a["eta2"][open_nodes]).max() > 0.01     # the tide has started
    assert a["uu2"][east].mean() < -0.02 and np.isfinite(a["eta2"]).all()


def test_zero_gradient_boundary_takes_the_interior_velocity(orc):
    """Zero normal velocity gradient (IBTYPE 40): each boundary node's
    velocity is the one interpolated at its fictitious interior node
    (mesh.F:2434-2512, momentum.F:1157-1174), the fictitious node lies in
    its element (interpolation factors in [0, 1], summing to 1), and the
    tide flows out through the boundary."""
    from adcirc_b200 import model
    c = model.channel_case(zero_gradient=True, prep=orc.mesh_prep())
    a = c.arrays
    nv = c.sizes["nvel"]
    j = np.where(a["lbcodei"][:nv] == 40)[0]
    f = np.stack([a["zngif1"][j], a["zngif2"][j], a["zngif3"][j]])
    assert j.size == 41 and (f >= -1e-12).all() and np.allclose(f.sum(axis=0), 1.0, atol=1e-12)
    om = orc.OracleModel(c)
    om.run(1, 1500)
    om.close()
    e = a["nelezng"][j] - 1
    nm = a["nm"] - 1
    for comp in ("uu2", "vv2"):
        v = a[comp]
        interp = sum(v[nm[e, k]] * f[k] for k in range(3))
        assert np.allclose(v[a["nbv"][j] - 1], interp, rtol=0, atol=1e-15)
    east = a["x"] > 59.9e3
    assert a["uu2"][east].mean() > 0.02


def test_external_barrier_outflow_follows_the_weir_formula(orc):
    """IBTYPE 13 (external barrier, no tangential slip): the normal velocity
    at each boundary node is QN2/H2 with QN2 the supercritical weir outflow
    RampIntFlux * BARLANCFSP * R * sqrt(R g), R = 2/3 of the head over the
    crest at the start of the step, once R exceeds BARMIN = 0.04 m
    (weir_boundary.F90:1751-1759, momentum.F:846-856); below it, none."""
    from adcirc_b200 import model
    case = model.channel_case(barrier=-0.05, barrier_type=13)
    a = case.arrays
    lbc = a["lbcodei"]
    ent = np.nonzero(lbc == 13)[0]
    assert ent.size > 30
    nodes = a["nbv"][ent] - 1
    g = case.params["g"]
    om = orc.OracleModel(case)
    flowing = dry_steps = 0
    for it in range(1, 1401):
        head = a["eta2"][nodes].copy()          # ETA2 when the step starts
        om.step(it)
        st = case.schedule.step(it)
        R = 2.0 * (head - a["barlanht"][ent]) / 3.0
        q = np.where(R > 0.04, -st.rampintflux * a["barlancfsp"][ent] * R * np.sqrt(np.maximum(R, 0) * g),
                     0.0)
        wet = a["nodecode"][nodes] == 1
        want = -q / a["h2"][nodes]
        assert np.array_equal(a["uu2"][nodes][wet], want[wet]), it
        flowing += int((R > 0.04).any())
        dry_steps += int((R <= 0.04).all())
    om.close()
    assert flowing > 100 and dry_steps > 100


def test_levee_overtopping_floods_the_polder(orc):
    """An internal barrier (IBTYPE 4) with its crest at datum between the
    tidal channel and a dry polder: once the tide stands BARMIN over the
    crest, water crosses the barrier (weir_boundary.F90:1775-1942) and the
    receiving nodes wet the polder through NIBCNT (wetdry.F:813-816,
    1086-1090); the polder wets from the barrier outward.  With a crest
    10 m high nothing crosses."""
    from adcirc_b200 import model
    wet = {}
    for crest in (0.0, 10.0):
        case = model.channel_case(levee=crest, amp=2.0)
        a = case.arrays
        east = a["x"] > 30.0e3 + 1.0
        om = orc.OracleModel(case)
        first = None
        for k in range(10):
            om.run(1 + 100 * k, 100)
            if first is None and a["nodecode"][east].any():
                first = a["x"][east & (a["nodecode"] == 1)].max()
        om.close()
        wet[crest] = int(a["nodecode"][east].sum())
        if crest == 0.0:
            # within two element columns (0.5 km each) of the barrier
            assert first is not None and first <= 31.0e3 + 1.0
    assert wet[0.0] > 100 and wet[10.0] == 0


def test_barrier_pipe_floods_the_polder(orc):
    """A barrier too high to overtop (10 m) with a 1 m pipe under it (IBTYPE
    5, crown 0.5 m below datum): the pipe's discharge (weir_boundary.F90:
    2469-2579) floods the polder; with the crown 10 m up nothing crosses."""
    from adcirc_b200 import model
    wet = {}
    for crown in (-0.5, 10.0):
        case = model.channel_case(levee=10.0, levee_type=5, pipe=(crown, 1.0, 1.0), amp=2.0)
        a = case.arrays
        om = orc.OracleModel(case)
        om.run(1, 1000)
        om.close()
        wet[crown] = int(a["nodecode"][a["x"] > 30.0e3 + 1.0].sum())
    assert wet[-0.5] > 100 and wet[10.0] == 0
