"""adc_jcg_noalloc: the jcg entry point that allocates no device memory.

Some callers cannot let a library call cudaMalloc: a host that owns every
device byte through its own memory pool, or one that runs under a fixed
device-memory budget.  adc_jcg_noalloc serves them from a static device
array.  The GPU test checks that it returns what adc_jcg and the oracle's
jcg return for the same system, on two calls in a row (the second call
finds the first call's leftovers in the shared array), and that the
second call leaves the device's free memory unchanged.  The size checks
run on the host before any device work, so they need no GPU.  The file is
collected last, so a run that stops at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

REL_TOL = 1e-9     # solution tolerance used by the other JCG parity tests


def _system(seed):
    import oracle
    from adcirc_b200 import model
    case = model.channel_case()
    om = oracle.OracleModel(case)
    for it in range(1, 3):
        om.step(it)
    om.close()
    a = case.arrays
    n = case.sizes["np"]
    rng = np.random.default_rng(seed)
    return (n, case.sizes["mnei"], a["neitab"].copy(order="F"), a["coef"].copy(order="F"),
            rng.standard_normal(n), 1e-3 * rng.standard_normal(n))


def _call(fn, n, mnei, jcoef, coef, rhs, u, iparm, rparm):
    from adcirc_b200._lib import dp_, ip_, ptr
    nw = 4 * n + 4 * int(iparm[0])
    wksp = np.zeros(nw)
    iwksp = np.zeros(3 * n, np.int32)
    ier = C.c_int(-1)
    fn(C.byref(C.c_int(n)), C.byref(C.c_int(n)), C.byref(C.c_int(mnei)), ptr(jcoef, ip_),
       ptr(coef, dp_), ptr(rhs, dp_), ptr(u, dp_), ptr(iwksp, ip_), C.byref(C.c_int(nw)),
       ptr(wksp, dp_), ptr(iparm, ip_), ptr(rparm, dp_), C.byref(ier))
    return ier.value


def _run(lib, fn, sysargs):
    from adcirc_b200._lib import dp_, ip_, ptr
    n, mnei, jc, cf, rhs, u0 = sysargs
    jcoef, coef, r, u = jc.copy(order="F"), cf.copy(order="F"), rhs.copy(), u0.copy()
    iparm = np.zeros(12, np.int32)
    rparm = np.zeros(12)
    lib.adc_dfault(ptr(iparm, ip_), ptr(rparm, dp_))
    iparm[0] = 200
    rparm[0] = 1e-10
    lib.adc_jcg_reset()
    ier = _call(fn, n, mnei, jcoef, coef, r, u, iparm, rparm)
    return ier, u, coef, jcoef, r, iparm, rparm


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _run_oracle(sysargs):
    import oracle
    n, mnei, jc, cf, rhs, u0 = sysargs
    jcoef, coef, r, u = jc.copy(order="F"), cf.copy(order="F"), rhs.copy(), u0.copy()
    iparm, rparm = oracle.dfault()
    iparm[0] = 200
    rparm[0] = 1e-10
    oracle.load().orc_itpack_reset()
    ier = oracle.jcg(n, n, mnei, jcoef, coef, r, u, iparm, rparm)
    return ier, u, coef, jcoef, r, iparm, rparm


@pytest.mark.gpu
def test_noalloc_matches_jcg_twice(lib):
    import torch
    import oracle  # noqa: F401  (builds the checker used to make the systems)
    for k, seed in enumerate((11, 12)):
        sysargs = _system(seed)
        ref = _run(lib, lib.adc_jcg, sysargs)
        orc = _run_oracle(sysargs)
        free0 = torch.cuda.mem_get_info()[0]
        got = _run(lib, lib.adc_jcg_noalloc, sysargs)
        free1 = torch.cuda.mem_get_info()[0]
        if k == 1:   # the first call may load the module holding the array
            assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
        assert ref[0] == 0 and got[0] == 0 and orc[0] == 0, (ref[0], got[0], orc[0])
        assert got[5][0] == orc[5][0], "iteration count vs oracle"
        assert _rel(got[1], orc[1]) <= REL_TOL
        assert _rel(got[2], orc[2]) <= 1e-13
        assert np.array_equal(got[3], orc[3])
        assert got[5][0] == ref[5][0], "iteration count"
        assert _rel(got[1], ref[1]) <= REL_TOL
        assert _rel(got[2], ref[2]) <= 1e-13
        assert np.array_equal(got[3], ref[3])
        assert _rel(got[4], ref[4]) <= 1e-13
        assert abs(got[6][1] - ref[6][1]) <= 1e-12 * max(abs(ref[6][1]), 1.0)


def _call_sized(lib, n, mnei, itmax):
    """adc_jcg_noalloc on a system whose size the host check rejects before
    any device work (the arrays are never read)."""
    from adcirc_b200 import _lib
    iparm = np.array([itmax, -1, 0, 6, 0, 1, 1, 0, -2, 0, 0, 3], np.int32)
    rparm = np.zeros(12)
    z = np.zeros(1)
    zi = np.zeros(1, np.int32)
    ier = C.c_int(0)
    lib.adc_jcg_noalloc(C.byref(C.c_int(n)), C.byref(C.c_int(n)), C.byref(C.c_int(mnei)),
                        _lib.ptr(zi, _lib.ip_), _lib.ptr(z, _lib.dp_), _lib.ptr(z, _lib.dp_),
                        _lib.ptr(z, _lib.dp_), _lib.ptr(zi, _lib.ip_), C.byref(C.c_int(10 ** 8)),
                        _lib.ptr(z, _lib.dp_), _lib.ptr(iparm, _lib.ip_),
                        _lib.ptr(rparm, _lib.dp_), C.byref(ier))
    return ier.value


def test_noalloc_rejects_oversize(lib):
    from adcirc_b200 import _lib
    assert _call_sized(lib, 2_000_000, 16, 10) == 905
    assert "static scratch" in _lib.last_error()


def test_noalloc_rejects_near_cap_with_large_itmax(lib):
    """16,001 rows of 100 slots: the 31 padding rows of the last slice and a
    3,000-iteration CG tridiagonal push the exact layout past 32 MiB, though
    the per-row estimate alone stays under it."""
    from adcirc_b200 import _lib
    assert 16_001 * (20 * 99 + 112) + 65536 < 32 << 20
    assert _call_sized(lib, 16_001, 100, 3000) == 905
    assert "static scratch" in _lib.last_error()
    assert _call_sized(lib, 1000, 16, 5000) == 905    # above the scalar block's ITMAX
