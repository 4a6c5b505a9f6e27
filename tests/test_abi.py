"""The C-ABI library builds, loads and exports every symbol of include/adcgpu.h."""
import ctypes as C

import numpy as np


def test_exports_all_declared_symbols(lib):
    from adcirc_b200 import _lib
    names = _lib.exported_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_dfault_matches_reference_defaults(lib, orc):
    from adcirc_b200._lib import dp_, ip_, ptr
    ip1 = np.zeros(12, np.int32)
    rp1 = np.zeros(12)
    lib.adc_dfault(ptr(ip1, ip_), ptr(rp1, dp_))
    ip2, rp2 = orc.dfault()
    assert np.array_equal(ip1, ip2) and np.array_equal(rp1, rp2)
    assert ip1[0] == 100 and ip1[8] == -2 and rp1[0] == 5e-6 and rp1[7] == 128 * 2.0 ** -52


def test_jcg_argument_errors_without_gpu(lib):
    """Argument checks that return before any device work (itpackv.F:239-243)."""
    from adcirc_b200._lib import dp_, ip_, ptr
    n = C.c_int(0)
    iparm = np.array([10, -1, 0, 6, 0, 1, 1, 0, -2, 0, 0, 3], np.int32)
    rparm = np.zeros(12)
    ier = C.c_int(-7)
    z = np.zeros(4)
    zi = np.zeros(4, np.int32)
    lib.adc_jcg(C.byref(n), C.byref(C.c_int(1)), C.byref(C.c_int(1)), ptr(zi, ip_), ptr(z, dp_),
                ptr(z, dp_), ptr(z, dp_), ptr(zi, ip_), C.byref(C.c_int(4)), ptr(z, dp_),
                ptr(iparm, ip_), ptr(rparm, dp_), C.byref(ier))
    assert ier.value == 11
    # zero diagonal -> 401 (itpackv.F:2370-2376)
    n1 = C.c_int(2)
    jcoef = np.array([1, 2], np.int32)
    coef = np.array([0.0, 1.0])
    lib.adc_jcg(C.byref(n1), C.byref(n1), C.byref(C.c_int(1)), ptr(jcoef, ip_), ptr(coef, dp_),
                ptr(z, dp_), ptr(z, dp_), ptr(zi, ip_), C.byref(C.c_int(100)), ptr(z, dp_),
                ptr(iparm, ip_), ptr(rparm, dp_), C.byref(ier))
    assert ier.value == 401


def test_bind_fails_cleanly_without_device(lib):
    """On a host without a GPU, binding reports ADC_ERR_CUDA instead of crashing."""
    import torch
    if torch.cuda.is_available():
        return
    from adcirc_b200 import model
    case = model.channel_case()
    try:
        model.GpuModel(case)
    except model.AdcError as e:
        assert "status -3" in str(e)
    else:
        raise AssertionError("bind succeeded without a device")
