"""Comparison of two ADCIRC ASCII output files (fort.61-64 and the like) with
the semantics of the reference's acceptance comparator,
util/adcircResultsComparison.F90, so that results of this library (written
with adcirc_io.Fort6x) can be checked against a reference adcirc run made
wherever a Fortran compiler exists.

- Format (checkFormat_fullFormatAscii / checkFormat_sparseFormatAscii,
  :499-543): the third line of a full-format file holds "time it", of a
  sparse-format file "time it nnondefault default".
- Records (readNextSnapFullAscii / readNextSnapSparseAscii, :659-697): full
  records list every node; sparse records the non-default nodes, the rest
  take the default value.
- Per record and value column (compareData, :718-758): with `wetdry`, nodes
  where either file holds a value <= -9999 (dry) are skipped; d = a - b;
  ndiff counts |d| > eps (eps = epsilon(1d0)), nerror counts |d| > tolerance
  (default 1e-5), maxdiff is the signed d of largest |d| above eps, and
  avgdiff the sum of d over all nodes (skipped ones included) divided by
  the node count.

    python -m adcirc_b200.compare fort.63 ref/fort.63 [-t 1e-5] [-w]

exits 1 when any value differs by more than the tolerance.
"""
from __future__ import annotations

import argparse
import dataclasses
import sys

import numpy as np

EPS = float(np.finfo(np.float64).eps)   # epsilon(1d0)


@dataclasses.dataclass
class OutputFile:
    header: str
    numsnaps: int                 # as the header states it
    numnodes: int
    numvalues: int
    times: list                   # per record: (time [s], time step)
    data: list                    # per record: (numnodes, numvalues) float64


def _floats(line: str):
    return [float(t.replace("D", "E").replace("d", "e")) for t in line.replace(",", " ").split()]


def read_output(path) -> OutputFile:
    """Reads a full- or sparse-format ASCII output file."""
    with open(path) as f:
        lines = f.read().splitlines()
    if len(lines) < 2:
        raise ValueError(f"{path}: no header")
    h = lines[1].split()
    numsnaps, numnodes, numvalues = int(h[0]), int(h[1]), int(h[4])
    sparse = len(lines) > 2 and len(lines[2].split()) >= 4
    times, data = [], []
    k = 2
    while k < len(lines):
        if not lines[k].strip():
            k += 1
            continue
        head = _floats(lines[k])
        k += 1
        rec = np.zeros((numnodes, numvalues))
        if sparse:
            nnon, default = int(head[2]), head[3]
            rec[:] = default
            for _ in range(nnon):
                v = _floats(lines[k])
                k += 1
                rec[int(v[0]) - 1, :] = v[1:1 + numvalues]
        else:
            for i in range(numnodes):
                v = _floats(lines[k])
                k += 1
                rec[i, :] = v[1:1 + numvalues]
        times.append((head[0], int(head[1])))
        data.append(rec)
    return OutputFile(lines[0], numsnaps, numnodes, numvalues, times, data)


@dataclasses.dataclass
class RecordDiff:
    ndiff: int
    nerror: int
    avgdiff: float
    maxdiff: float


def compare_data(a: np.ndarray, b: np.ndarray, tolerance: float = 1.0e-5,
                 wetdry: bool = False) -> RecordDiff:
    """compareData (adcircResultsComparison.F90:718-758) for one column."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    keep = np.ones(a.shape, bool)
    if wetdry:
        keep = ~((a <= -9999.0) | (b <= -9999.0))
    d = (a - b)[keep]
    ad = np.abs(d)
    ndiff = int(np.sum(ad > EPS))
    nerror = int(np.sum(ad > tolerance))
    maxdiff = 0.0
    for x in d[ad > EPS]:   # the first d of the largest |d|, in node order
        if abs(x) > abs(maxdiff):
            maxdiff = float(x)
    avgdiff = float(np.sum(d)) / a.size
    return RecordDiff(ndiff, nerror, avgdiff, maxdiff)


def compare_files(path1, path2, tolerance: float = 1.0e-5, wetdry: bool = False):
    """Per record and value column the RecordDiff of the two files; raises
    ValueError when their node or value counts differ."""
    f1, f2 = read_output(path1), read_output(path2)
    if (f1.numnodes, f1.numvalues) != (f2.numnodes, f2.numvalues):
        raise ValueError("the files hold different node or value counts")
    n = min(len(f1.data), len(f2.data))
    return [[compare_data(f1.data[s][:, j], f2.data[s][:, j], tolerance, wetdry)
             for j in range(f1.numvalues)] for s in range(n)]


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("file1")
    ap.add_argument("file2")
    ap.add_argument("-t", "--tolerance", type=float, default=1.0e-5)
    ap.add_argument("-w", "--wetdry", action="store_true",
                    help="skip nodes that either file marks dry (<= -9999)")
    args = ap.parse_args(argv)
    res = compare_files(args.file1, args.file2, args.tolerance, args.wetdry)
    worst = 0
    for s, cols in enumerate(res):
        for j, r in enumerate(cols):
            print(f"record {s + 1} value {j + 1}: ndiff {r.ndiff} nerror {r.nerror} "
                  f"avgdiff {r.avgdiff:.6e} maxdiff {r.maxdiff:.6e}")
            worst = max(worst, r.nerror)
    return 1 if worst else 0


if __name__ == "__main__":
    sys.exit(main())
