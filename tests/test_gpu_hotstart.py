"""Hotstart dump/load (adc_hotstart_write / adc_hotstart_read): a run
resumed from a hotstart continues bit for bit, the resume test of the
reference's hotstart path (write_output.F:4429-5582, hstart.F:47-2048)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("eta1", "eta2", "etas", "uu2", "vv2", "qx2", "qy2", "h2", "tk", "totalarea", "coef",
          "wsx2", "pr2", "nodecode", "noff", "mju")


def _resume_equal(case_fn, n, prec, tmp_path, use_run):
    from adcirc_b200 import model
    base = case_fn()
    full, first, resumed = base.clone(), base.clone(), base.clone()
    a = model.GpuModel(full, prec=prec)
    b = model.GpuModel(first, prec=prec)
    h = n // 2
    if use_run:
        a.run(1, n)
        b.run(1, h)
    else:
        for it in range(1, n + 1):
            a.step(it)
        for it in range(1, h + 1):
            b.step(it)
    path = tmp_path / "hot.adc"
    b.hotstart_write(path)
    b.close()
    c = model.GpuModel(resumed, prec=prec)   # fresh context, original arrays
    c.hotstart_read(path)
    if use_run:
        c.run(h + 1, n - h)
    else:
        for it in range(h + 1, n + 1):
            c.step(it)
    a.sync_to_host()
    c.sync_to_host()
    a.close()
    c.close()
    for f in FIELDS:
        assert np.array_equal(full.arrays[f], resumed.arrays[f]), f


def test_resume_channel_vortex(lib, tmp_path):
    from adcirc_b200 import model
    _resume_equal(lambda: model.channel_case(vortex=True), 80, 0, tmp_path, use_run=False)


def test_resume_beach_wetdry_graph(lib, tmp_path):
    from adcirc_b200 import model
    _resume_equal(model.beach_case, 300, 0, tmp_path, use_run=True)


def test_resume_mixed_warm(lib, tmp_path):
    from adcirc_b200 import model
    _resume_equal(lambda: model.channel_case(vortex=True), 60, 1 | 2, tmp_path, use_run=True)


def test_hotstart_rejects_other_mesh_or_mode(lib, tmp_path):
    from adcirc_b200 import model
    g = model.GpuModel(model.channel_case())
    g.run(1, 5)
    path = tmp_path / "hot.adc"
    g.hotstart_write(path)
    g.close()
    other = model.GpuModel(model.beach_case())
    with pytest.raises(model.AdcError):
        other.hotstart_read(path)
    other.close()
    mixed = model.GpuModel(model.channel_case(), prec=1)
    with pytest.raises(model.AdcError):
        mixed.hotstart_read(path)
    mixed.close()
    bad = tmp_path / "bad.adc"
    bad.write_bytes(b"not a hotstart file")
    g2 = model.GpuModel(model.channel_case())
    with pytest.raises(model.AdcError):
        g2.hotstart_read(bad)
    g2.close()


def test_resume_channel_river(lib, tmp_path):
    from adcirc_b200 import model
    _resume_equal(lambda: model.channel_case(river=0.5), 80, 0, tmp_path, use_run=True)


def test_resume_series(lib, tmp_path):
    """fort.19 and fort.20 series: the record pair, its times and the ratio
    travel in the hotstart file."""
    from adcirc_b200 import model
    _resume_equal(lambda: model.channel_case(river=0.5, elev_series=150.0, flux_series=300.0,
                                             series_hours=1.0), 240, 0, tmp_path, use_run=True)


def test_resume_zero_gradient(lib, tmp_path):
    """Zero-normal-gradient entries keep QN0 from the step before the dump."""
    from adcirc_b200 import model
    _resume_equal(lambda: model.channel_case(zero_gradient=True), 80, 0, tmp_path, use_run=True)


def test_resume_levee(lib, tmp_path):
    """An internal barrier between channel and polder: the run resumed while
    the polder floods continues bit for bit."""
    from adcirc_b200 import model
    _resume_equal(lambda: model.channel_case(levee=0.0, amp=2.0), 800, 0, tmp_path, use_run=True)
