"""GPU parity on the benchmark mesh and over long runs.

* The ~600k-node storm-surge mesh (the workload bench.py times) from cold
  start: the resident JCG variant at full size (hundreds of row blocks,
  halo lists, block-local uint16 columns, staged slices), the incremental
  GWCE matrix rebuild and the wet/dry passes, against the oracle.
* A mid-storm window on the same mesh: the plain FP64 path runs to 18 h
  (the vortex makes landfall at about 19 h), and the oracle then continues
  from that state (arrays plus the module scalars of adc_get_scalars) step
  for step beside the GPU, through steps with W1 wetting events, matrix
  rebuilds (NCChange > 0) and the moving front.
* The 4,961-node tidal channel over its full 2-day run (34,560 steps).

Tolerances as in test_gpu_parity: fields within 1e-9 relative, identical
JCG iteration counts every step, NODECODE/NOFF/MJU bit for bit.
"""
import copy

import numpy as np
import pytest

from test_gpu_parity import FIELDS, REL_TOL, _check, _rel, oracle_and_gpu_cases

pytestmark = pytest.mark.gpu

SURGE_NODES = 600_000
MID_STORM_HOURS = 18
WINDOW = 16


@pytest.fixture(scope="module")
def surge_raw():
    from adcirc_b200 import meshgen
    return meshgen.surge_mesh(seed=2024, target_nodes=SURGE_NODES)


def _surge_pair(raw):
    from adcirc_b200 import model
    return oracle_and_gpu_cases(lambda **k: model.surge_case(raw=copy.deepcopy(raw), **k))


def _compare_state(c0, cg):
    a, b = c0.arrays, cg.arrays
    errs = {f: _rel(b[f], a[f]) for f in FIELDS}
    bad = {f: e for f, e in errs.items() if not e <= REL_TOL}
    assert not bad, f"fields beyond {REL_TOL}: {bad}"
    for f in ("nodecode", "nnodecode", "noff", "mju"):
        nm = int(np.sum(a[f] != b[f]))
        assert nm == 0, f"{f}: {nm} mismatches"
    return errs


def test_surge_cold_start(lib, orc, surge_raw):
    import oracle
    from adcirc_b200 import model
    c0, cg = _surge_pair(surge_raw)
    assert 590_000 <= c0.sizes["np"] <= 610_000
    n = 20
    om = oracle.OracleModel(c0)
    its_o = om.run(1, n)
    gm = model.GpuModel(cg)
    its_g, _ = gm.run(1, n)
    gm.sync_to_host()
    gm.close()
    om.close()
    _check(c0, cg, its_o, np.asarray(its_g))
    _compare_state(c0, cg)
    assert its_o.min() > 0


def test_surge_mid_storm_window(lib, orc, surge_raw):
    """Resume the oracle from the GPU's state at 18 h and step both."""
    import oracle
    from adcirc_b200 import model
    c0, cg = _surge_pair(surge_raw)
    gm = model.GpuModel(cg)
    spd = int(round(3600.0 / cg.params["dt"]))
    it = 1
    for _ in range(MID_STORM_HOURS):
        gm.run(it, spd)
        it += spd
    gm.sync_to_host()
    sc = gm.scalars()
    for k in model.STATE_F64 + model.STATE_I32:
        np.copyto(c0.arrays[k], cg.arrays[k])
    om = oracle.OracleModel(c0)
    om.set_scalars(sc)
    its_o, its_g, w1, ncc = [], [], [], []
    for k in range(WINDOW):
        oo = om.step(it + k)
        go = gm.step(it + k)
        its_o.append(oo.numitr)
        its_g.append(go.numitr)
        w1.append((oo.n_w1_events, go.n_w1_events))
        ncc.append((oo.ncchange, go.ncchange))
    gm.sync_to_host()
    gm.close()
    om.close()
    assert [x[0] for x in w1] == [x[1] for x in w1], f"W1 event counts differ: {w1}"
    assert [x[0] for x in ncc] == [x[1] for x in ncc], f"NCChange differs: {ncc}"
    _check(c0, cg, np.asarray(its_o), np.asarray(its_g))
    _compare_state(c0, cg)
    # the window is the one that matters: fronts move and the matrix is rebuilt
    assert sum(x[0] for x in w1) > 0, f"no W1 wetting events in the window: {w1}"
    assert all(x[0] > 0 for x in ncc), f"steps without a matrix rebuild: {ncc}"
    assert sc["vortex_counter"] >= 1


def test_channel_two_day_run(lib, orc):
    """The tidal channel for its whole 2-day run: per-step iteration counts
    and the final state.  The run has the advective terms off (fort.15
    NOLICA = NOLICAT = 0, which the channel configuration leaves open): with
    them on, velocities at the corner where the open boundary meets the
    north shore grow from hour 12 and the run diverges by hour 16, in the
    oracle and on the GPU alike, with identical iteration counts.  The
    shorter channel runs and the beach, river and surge cases keep the
    advective terms on."""
    import oracle
    from adcirc_b200 import model
    c0, cg = oracle_and_gpu_cases(lambda **k: model.channel_case(ifnlct=0, ifnlcat=0, **k))
    n = int(round(2 * 86400 / c0.params["dt"]))
    om = oracle.OracleModel(c0)
    its_o = om.run(1, n)
    om.close()
    gm = model.GpuModel(cg)
    its_g, _ = gm.run(1, n)
    gm.sync_to_host()
    gm.close()
    its_g = np.asarray(its_g)
    mism = int(np.sum(its_o != its_g))
    assert mism == 0, f"iteration counts differ in {mism} of {n} steps"
    _check(c0, cg, its_o, its_g)
    assert np.abs(c0.arrays["eta2"]).max() > 0.1   # the tide is still running
