"""The output comparator (adcirc_b200.compare) against hand-made files: the
semantics of the reference's util/adcircResultsComparison.F90 (tolerance,
epsilon-level differences, dry-node skipping, sparse records)."""
import numpy as np

from adcirc_b200 import adcirc_io, compare


def _write(path, recs, v2=False, nodecode=None):
    n = recs[0][0].size
    f = adcirc_io.Fort6x(path, n, 2 if v2 else 1, 60.0, 12, len(recs))
    for k, r in enumerate(recs):
        f.append(60.0 * (k + 1), 12 * (k + 1), r[0], r[1] if v2 else None,
                 nodecode=None if nodecode is None else nodecode[k])


def test_full_format_counts(lib, tmp_path):
    a = np.linspace(-0.5, 0.5, 7)
    b = a.copy()
    b[2] += 2e-5          # an error at the default tolerance
    b[4] += 1e-9          # a difference, not an error
    _write(tmp_path / "a.63", [(a, None), (a, None)])
    _write(tmp_path / "b.63", [(a, None), (b, None)])
    f = compare.read_output(tmp_path / "b.63")
    assert (f.numnodes, f.numvalues, len(f.data)) == (7, 1, 2)
    assert f.times[1] == (120.0, 24)
    res = compare.compare_files(tmp_path / "a.63", tmp_path / "b.63")
    assert res[0][0].ndiff == 0 and res[0][0].nerror == 0 and res[0][0].maxdiff == 0.0
    r = res[1][0]
    assert r.ndiff == 2 and r.nerror == 1
    assert np.isclose(r.maxdiff, -2e-5, rtol=1e-9)
    assert compare.main([str(tmp_path / "a.63"), str(tmp_path / "b.63")]) == 1
    assert compare.main([str(tmp_path / "a.63"), str(tmp_path / "b.63"), "-t", "1e-4"]) == 0


def test_wetdry_skips_dry_nodes(lib, tmp_path):
    a = np.array([0.1, 0.2, 0.3, 0.4])
    b = np.array([0.1, 5.0, 0.3, 0.4])
    dry = np.array([1, 0, 1, 1], np.int32)
    _write(tmp_path / "a.63", [(a, None)], nodecode=[dry])     # node 2 written as -99999
    _write(tmp_path / "b.63", [(b, None)])
    plain = compare.compare_files(tmp_path / "a.63", tmp_path / "b.63")[0][0]
    skip = compare.compare_files(tmp_path / "a.63", tmp_path / "b.63", wetdry=True)[0][0]
    assert plain.nerror == 1 and skip.nerror == 0 and skip.avgdiff == 0.0


def test_velocity_columns_and_sparse_records(lib, tmp_path):
    u = np.array([0.0, 1.0, 2.0])
    v = np.array([0.5, 0.5, 0.5])
    _write(tmp_path / "full.64", [(u, v)], v2=True)
    sparse = tmp_path / "sparse.64"
    lines = (tmp_path / "full.64").read_text().splitlines()[:2]
    lines += ["  6.0000000000E+001  12  2  0.0", "  2  1.0  0.5", "  3  2.0  0.75"]
    sparse.write_text("\n".join(lines) + "\n")
    s = compare.read_output(sparse)
    assert np.array_equal(s.data[0], [[0.0, 0.0], [1.0, 0.5], [2.0, 0.75]])
    res = compare.compare_files(tmp_path / "full.64", sparse)[0]
    assert res[0].nerror == 0 and res[1].nerror == 2
