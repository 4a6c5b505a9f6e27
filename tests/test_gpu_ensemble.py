"""Batched ensembles (adc_ensemble_*): members stepped together in one
captured graph per time step give exactly what each member gives alone,
also after the JCG layout of a member changes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _members():
    """Three channel members with one step table: different tides and
    vortex tracks."""
    from adcirc_b200 import model
    cases = [model.channel_case(vortex=True), model.channel_case(vortex=True, amp=0.3),
             model.channel_case(vortex=True, amp=0.7)]
    cases[1].vortex = model.straight_track(20e3, 2e3, 70.0, 4.0, 950.0, 6.0, 1.3, hours=12.0,
                                           interval_h=3.0)
    cases[2].vortex = model.straight_track(40e3, 18e3, 250.0, 7.0, 930.0, 10.0, 1.3, hours=12.0,
                                           interval_h=3.0)
    return cases


def test_ensemble_equals_members_alone(lib):
    from adcirc_b200 import ensemble, model
    alone = _members()
    together = _members()
    its_alone = []
    for c in alone:
        g = model.GpuModel(c)
        its, _ = g.run(1, 120)
        g.sync_to_host()
        g.close()
        its_alone.append(np.asarray(its))
    ens = ensemble.Ensemble(together)
    its, ms = ens.run(60)
    its2, _ = ens.run(60)
    for m in ens.models:
        m.sync_to_host()
    ens.close()
    assert ms > 0
    for k, (a, b) in enumerate(zip(alone, together)):
        assert np.array_equal(np.concatenate([its[k], its2[k]]), its_alone[k]), k
        for f in ("eta2", "uu2", "vv2", "nodecode"):
            assert np.array_equal(a.arrays[f], b.arrays[f]), (k, f)


def test_ensemble_layouts_and_autotune(lib):
    """Changing the members' JCG row blocks keeps every member within the
    parity tolerance of its standalone run; the autotuner picks a layout."""
    from adcirc_b200 import ensemble, model
    alone = _members()
    for c in alone:
        g = model.GpuModel(c)
        g.run(1, 150)
        g.sync_to_host()
        g.close()
    cases = _members()
    ens = ensemble.Ensemble(cases)
    ens.run(20)
    best, res = ensemble.autotune(ens, steps=10, log=lambda *a: None)
    assert best in res and all(r["ms_per_step"] > 0 for r in res.values())
    ens.run(150 - ens.it + 1)
    for m in ens.models:
        m.sync_to_host()
    ens.close()
    for a, b in zip(alone, cases):
        e = np.abs(a.arrays["eta2"] - b.arrays["eta2"]).max() / np.abs(a.arrays["eta2"]).max()
        assert e <= 1e-9, e
        assert np.array_equal(a.arrays["nodecode"], b.arrays["nodecode"])
