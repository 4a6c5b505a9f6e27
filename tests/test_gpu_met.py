"""GPU parity of the NWS = 8 vortex forcing (adc_set_vortex) against the
oracle.  The met fields use CUDA's exp/pow/sin/cos/atan2 and the oracle
glibc's, so they agree to ~1e-15 rather than bit for bit; the coupled
model keeps the FP64 path's 1e-9 bound and identical JCG iteration counts.
"""
import ctypes as C

import numpy as np
import pytest

from test_gpu_parity import REL_TOL, _check, _pair, _rel, oracle_and_gpu_cases

pytestmark = pytest.mark.gpu


def test_vortex_fields_first_steps(lib, orc):
    import oracle
    from adcirc_b200 import model
    c0, cg = oracle_and_gpu_cases(lambda **k: model.channel_case(vortex=True, **k))
    o = oracle.OracleModel(c0)
    g = model.GpuModel(cg)
    for it in (1, 2, 3):
        o.step(it)
        g.step(it)
        g.sync_to_host()
        for f in ("wsx2", "wsy2", "pr2"):
            e = _rel(cg.arrays[f], c0.arrays[f])
            assert e < 1e-13, (it, f, e)
    g.close()
    o.close()


def test_vortex_channel_steps(lib, orc):
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(vortex=True, **k), 60)
    errs = _check(c0, cg, io, ig)
    # the storm must actually force the channel
    assert np.abs(c0.arrays["wsx2"]).max() > 1e-4
    assert max(errs.values()) <= REL_TOL


def test_vortex_graph_run(lib, orc):
    from adcirc_b200 import model
    c0, cg, io, ig = _pair(lambda **k: model.channel_case(vortex=True, **k), 150, use_run=True)
    _check(c0, cg, io, ig)


def test_vortex_track_end_is_reported(lib):
    """Past the last fix the reference terminates (nws08.F90:847-852); the
    library returns ADC_ERR_ARG from the step instead."""
    from adcirc_b200 import _lib, model
    case = model.channel_case(vortex=True)
    short = model.Vortex(case.vortex.fixes[:2].copy())
    short.fixes[1, 0] = 12.0
    case.vortex = short
    g = model.GpuModel(case)
    s = case.schedule
    out = _lib.AdcStepOut()
    assert lib.adc_timestep(g.h, C.byref(s.step(1)), C.byref(out)) == 0
    assert lib.adc_timestep(g.h, C.byref(s.step(2)), C.byref(out)) == 0
    rc = lib.adc_timestep(g.h, C.byref(s.step(3)), C.byref(out))
    assert rc == _lib.ADC_ERR_ARG and out.status == _lib.ADC_ERR_ARG
    g.close()


def test_set_vortex_rejects_bad_tracks(lib):
    from adcirc_b200 import model
    case = model.channel_case(vortex=True)
    g = model.GpuModel(case)
    for fixes in (case.vortex.fixes[:1], case.vortex.fixes[::-1]):
        v, arr = model.Vortex(fixes.copy()).struct()
        assert lib.adc_set_vortex(g.h, C.byref(v)) != 0
    g.close()
    # NWS = 0 in the bound parameters
    plain = model.channel_case()
    g = model.GpuModel(plain)
    v, arr = case.vortex.struct()
    assert lib.adc_set_vortex(g.h, C.byref(v)) != 0
    g.close()


def test_vortex_calm_period(lib, orc):
    """A track with a CALM line: no wind and the background pressure while it
    brackets the time (nws08.F90:588-601, 858-872), the storm after it,
    against the oracle over a graph-replayed run."""
    from test_oracle_met import calm_track_case
    c0, cg, io, ig = _pair(calm_track_case, 120, use_run=True)
    _check(c0, cg, io, ig)
    for f in ("wsx2", "wsy2", "pr2"):
        assert _rel(cg.arrays[f], c0.arrays[f]) < 1e-13, f
