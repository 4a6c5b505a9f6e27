"""GPU checks of the FP32 components (ADC_PREC_MIXED, ADC_F32_*) and of
the extrapolated initial guess (ADC_WARM_START).

These modes leave the reference's arithmetic on purpose, so they are held
to accuracy bounds against the FP64 path, not to bitwise parity: the
north-star bound max |d eta| <= 1 mm, and RMS |d u| reported beside it.
The channel is fully wet, so differences there measure precision alone
(no wetting/drying front amplifies them).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NSTEPS = 300


def _run(case, prec, n=NSTEPS):
    from adcirc_b200 import model
    g = model.GpuModel(case, prec=prec)
    its, _ = g.run(1, n)
    g.sync_to_host()
    stats = None
    if prec & 2:
        u, f = C.c_longlong(), C.c_longlong()
        g.lib.adc_warm_start_stats(g.h, C.byref(u), C.byref(f))
        stats = (u.value, f.value)
    g.close()
    return np.asarray(its), stats


def _diff(a, b):
    de = float(np.abs(a["eta2"] - b["eta2"]).max())
    du = float(np.sqrt(np.mean((a["uu2"] - b["uu2"]) ** 2 + (a["vv2"] - b["vv2"]) ** 2)))
    return de, du


@pytest.fixture(scope="module")
def fp64_channel(lib):
    from adcirc_b200 import model
    base = model.channel_case(vortex=True)
    ref = base.clone()
    its, _ = _run(ref, 0)
    return base, ref, its


@pytest.mark.parametrize("flags", [1, 4, 8, 16])
def test_fp32_components_within_1mm(lib, fp64_channel, flags):
    base, ref, its_ref = fp64_channel
    c = base.clone()
    its, _ = _run(c, flags)
    de, du = _diff(c.arrays, ref.arrays)
    assert np.isfinite(c.arrays["eta2"]).all()
    assert de <= 1e-3, f"flags {flags}: max|d eta| {de:.3e} m"
    assert du <= 1e-3, f"flags {flags}: RMS|d u| {du:.3e} m/s"
    # the FP32 matrix changes the solve by far less than its tolerance
    if flags == 8:
        assert de <= 1e-8
    # iterations stay those of the same tolerance
    assert abs(float(its.mean()) - float(its_ref.mean())) <= 1.0


def test_warm_start_same_tolerance(lib, fp64_channel):
    base, ref, its_ref = fp64_channel
    c = base.clone()
    its, (used, fallback) = _run(c, 2)
    assert used + fallback == NSTEPS
    assert used > NSTEPS // 2
    de, du = _diff(c.arrays, ref.arrays)
    # only the starting point of each solve differs; both stop at 1e-10
    assert de <= 1e-6 and du <= 1e-6
    assert its.mean() <= its_ref.mean()


def test_mixed_wetdry_runs(lib):
    """The beach case dries and floods: the mixed path must keep its
    wet/dry flags close to the FP64 path's (fronts are where precision
    shows first)."""
    from adcirc_b200 import model
    base = model.beach_case()
    ref, mix = base.clone(), base.clone()
    _run(ref, 0, 400)
    _run(mix, 1, 400)
    a, b = mix.arrays, ref.arrays
    assert np.isfinite(a["eta2"]).all()
    mism = int((a["nodecode"] != b["nodecode"]).sum())
    assert mism <= 0.02 * a["nodecode"].size, mism
