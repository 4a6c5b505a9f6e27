"""Known answers on the GPU path: volume conservation, the inflow mass
balance, mirror symmetry and the quarter-annulus analytic tide
(kat_cases.py), and the slope limiter (computeAlpha, wetdry.F:1561-1652)
with ALPHAL < 1 against the oracle."""
import numpy as np
import pytest

import kat_cases as K
from test_gpu_parity import _check, _rel, oracle_and_gpu_cases

pytestmark = pytest.mark.gpu


def test_gpu_closed_basin_conserves_volume(lib):
    from adcirc_b200 import model
    c = K.closed_basin()
    v0 = K.basin_volume(c)
    g = model.GpuModel(c)
    drift = []
    for k in range(8):
        g.run(1 + 50 * k, 50)
        g.sync_to_host()
        drift.append(K.basin_volume(c) - v0)
    g.close()
    assert np.abs(c.arrays["eta2"]).max() > 0.05
    assert max(abs(d) for d in drift) <= 1e-8 * v0, max(abs(d) for d in drift) / v0


def test_gpu_river_inflow_mass_balance(lib):
    from adcirc_b200 import model
    c = K.river_basin()
    g = model.GpuModel(c)
    g.run(1, 719)
    g.sync_to_host()
    v1 = K.basin_volume(c)
    g.run(720, 721)
    g.sync_to_host()
    v2 = K.basin_volume(c)
    g.close()
    q = K.inflow_volume(c, 720, 1441)
    assert abs((v2 - v1) - q) <= 1e-6 * q, ((v2 - v1) - q) / q


def test_gpu_mirror_symmetry(lib):
    from adcirc_b200 import model
    c = K.mirror_channel()
    g = model.GpuModel(c)
    g.run(1, 720)
    g.sync_to_host()
    g.close()
    asym = K.asymmetry(c)
    assert asym["eta"] <= 1e-12 and asym["u"] <= 1e-12 and asym["v"] <= 1e-9, asym


def test_slope_limiter_alphal(lib, orc):
    """A finite SLIM on the beach: computeAlpha limits the gravity term of
    wet elements near the front (ALPHAL down to ~0.02), which also marks
    those elements for the incremental matrix rebuild.  ALPHAL is a
    nonlinear function of the elevation gradient, and eta differs from the
    oracle's in the last bits (the JCG dot products sum in another order),
    so ALPHAL must match to the fields' 1e-9 every step, with the same
    elements limited, and the run as a whole as in every parity test."""
    import oracle
    from adcirc_b200 import model
    c0, cg = oracle_and_gpu_cases(lambda **k: model.beach_case(slim=1e-5, **k))
    om = oracle.OracleModel(c0)
    gm = model.GpuModel(cg)
    its_o, its_g, limited = [], [], 0
    for it in range(1, 401):
        its_o.append(om.step(it).numitr)
        its_g.append(gm.step(it).numitr)
        gm.sync_to_host()
        a0, ag = c0.arrays["alphal"], cg.arrays["alphal"]
        assert np.abs(ag - a0).max() <= 1e-9, (it, float(np.abs(ag - a0).max()))
        assert np.array_equal(a0 < 1.0, ag < 1.0), it
        limited += int((a0 < 1.0).any())
    gm.close()
    om.close()
    assert limited >= 100, limited
    assert c0.arrays["alphal"].min() <= 1.0
    _check(c0, cg, np.asarray(its_o), np.asarray(its_g))


def test_gpu_quarter_annulus_matches_the_analytic_tide(lib, orc):
    """The quarter-annular harbour (kat_cases): the GPU's periodic tide
    matches the closed-form solution as the oracle's does, and the two
    runs agree to the parity tolerance after five days."""
    import oracle
    from adcirc_b200 import model
    c0, cg = oracle_and_gpu_cases(lambda **k: model.quarter_annulus_case(**k))
    g = model.GpuModel(cg)

    def run(it, n):
        g.run(it, n)
        g.sync_to_host()
    amp, ph = K.harmonic_m2(run, cg)
    g.close()
    a_err, p_err = K.annulus_errors(cg, amp, ph)
    assert a_err <= 5e-3 and p_err <= 0.5, (a_err, p_err)
    om = oracle.OracleModel(c0)
    it_end = int(5.0 * 86400.0 / c0.params["dt"]) + 2 * int(round(model.M2_PERIOD / c0.params["dt"]))
    om.run(1, it_end)
    om.close()
    assert _rel(cg.arrays["eta2"], c0.arrays["eta2"]) <= 1e-9
