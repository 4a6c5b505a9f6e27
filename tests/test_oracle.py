"""CPU checks of the oracle and of the host-side mesh tables.

No golden vectors exist for this path in the reference, so the oracle is
pinned by known answers: lake at rest, JCG against a direct sparse solve,
NeiTab/CSR_POSITION invariants, and conservation of the wet area.
"""
import math

import numpy as np
import pytest


def test_mesh_tables_channel(lib):
    from adcirc_b200 import model
    case = model.channel_case()
    a, s = case.arrays, case.sizes
    np_, ne = s["np"], s["ne"]
    assert (np_, ne) == (4961, 9600)
    assert np.all(a["areas"] > 0)
    assert math.isclose(a["areas"].sum() / 2.0, 60e3 * 20e3, rel_tol=1e-12)
    nt, nn = a["neitab"], a["nneigh"]
    x, y = a["x"], a["y"]
    for i in range(0, np_, 97):
        assert nt[i, 0] == i + 1
        nbr = nt[i, 1:nn[i]] - 1
        ang = []
        for j in nbr:
            dx, dy = x[j] - x[i], y[j] - y[i]
            t = math.degrees(math.acos(dx / math.hypot(dx, dy)))
            ang.append(360.0 - t if dy > 0 else t)
        assert all(ang[k] < ang[k + 1] for k in range(len(ang) - 1))
        for j in nbr:   # symmetric neighbour relation
            assert i + 1 in nt[j, 1:nn[j]]
    nm, cp = a["nm"] - 1, a["csr_position"]
    for e in range(0, ne, 31):
        for k in range(3):
            others = [nm[e, (k + 1) % 3], nm[e, (k + 2) % 3]]
            got = {nt[nm[e, k], cp[e, k, l] - 1] - 1 for l in range(2)}
            assert got == set(others)


def test_coldstart_product_matches_oracle(lib, orc):
    import ctypes as C
    from adcirc_b200 import model
    c1 = model.beach_case()
    c2 = c1.clone()
    for k in ("eta1", "eta2"):
        c2.arrays[k][:] = 0.0
    om = orc.OracleModel(c2)
    orc.load().orc_coldstart(C.byref(om.p), C.byref(om.a))
    for k in ("nodecode", "nnodecode", "noff", "mju"):
        assert np.array_equal(c1.arrays[k], c2.arrays[k]), k
    for k in ("eta1", "eta2", "totalarea"):
        assert np.array_equal(c1.arrays[k], c2.arrays[k]), k
    assert (c1.arrays["nodecode"] == 0).sum() > 0


def test_lake_at_rest_oracle(orc):
    from adcirc_b200 import model
    case = model.channel_case(amp=0.0)
    om = orc.OracleModel(case)
    its = om.run(1, 20)
    a = case.arrays
    assert np.all(a["eta2"] == 0.0) and np.all(a["uu2"] == 0.0) and np.all(its == 0)


def test_jcg_matches_direct_solve(orc):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    from adcirc_b200 import model
    case = model.channel_case()
    om = orc.OracleModel(case)
    om.step(1)
    om.close()
    a, s = case.arrays, case.sizes
    n, mnei = s["np"], s["mnei"]
    coef, nt = a["coef"].copy(order="F"), a["neitab"].copy(order="F")
    rows, cols, vals = [], [], []
    for j in range(mnei):
        m = nt[:, j] > 0
        rows.append(np.nonzero(m)[0])
        cols.append(nt[m, j] - 1)
        vals.append(coef[m, j])
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    rng = np.random.default_rng(3)
    b = rng.standard_normal(n)
    xref = spl.spsolve(A.tocsc(), b)
    iparm, rparm = orc.dfault()
    iparm[0] = 200
    rparm[0] = 1e-12
    u = np.zeros(n)
    rhs = b.copy()
    ier = orc.jcg(n, n, mnei, nt, coef, rhs, u, iparm, rparm)
    assert ier == 0 and iparm[0] > 0
    assert np.abs(u - xref).max() <= 1e-9 * np.abs(xref).max()
    # the matrix comes back unscaled up to rounding drift
    assert np.abs(coef - a["coef"]).max() <= 1e-12 * np.abs(a["coef"]).max()


def test_jcg_nonconvergence_overwrites_zeta(orc):
    """itpackv.F:389-395: ier = 13 and rparm(1) = stptst when itmax is hit."""
    from adcirc_b200 import model
    case = model.channel_case()
    om = orc.OracleModel(case)
    om.step(1)
    om.close()
    a, s = case.arrays, case.sizes
    n, mnei = s["np"], s["mnei"]
    iparm, rparm = orc.dfault()
    iparm[0] = 2
    rparm[0] = 1e-10
    u = np.zeros(n)
    rhs = np.random.default_rng(1).standard_normal(n)
    ier = orc.jcg(n, n, mnei, a["neitab"].copy(order="F"), a["coef"].copy(order="F"), rhs, u,
                  iparm, rparm)
    assert ier == 13 and iparm[0] == 2 and rparm[0] > 1e-10


def test_oracle_deterministic(orc):
    from adcirc_b200 import model
    res = []
    for _ in range(2):
        case = model.beach_case()
        om = orc.OracleModel(case)
        om.run(1, 50)
        res.append(case.arrays["eta2"].copy())
    assert np.array_equal(res[0], res[1])


def test_beach_wets_and_dries(orc):
    from adcirc_b200 import model
    case = model.beach_case()
    om = orc.OracleModel(case)
    wet0 = int(case.arrays["nodecode"].sum())
    seen = set()
    for it in range(1, 601):
        o = om.step(it)
        seen.add(int(case.arrays["nodecode"].sum()))
    assert len(seen) > 3, "the wet area never changed"
    assert min(seen) >= 0 and max(seen) <= case.sizes["np"]
    assert wet0 > 0


@pytest.mark.parametrize("river_type", [2, 22])
def test_river_inflow_oracle(orc, river_type):
    """With no tide, a steady inflow of q m^2/s per unit width through the
    east end raises the water and drives the flow at the boundary to about
    -q/H (a specified-flux boundary, timestep.F:861-880, gwce.F:1737-1834)."""
    from adcirc_b200 import model
    c = model.channel_case(amp=0.0, river=0.5, river_type=river_type)
    o = orc.OracleModel(c)
    for it in range(1, 401):
        o.step(it)
    o.close()
    a = c.arrays
    east = a["x"] > 59.9e3
    u = a["uu2"][east].mean()
    assert -0.12 < u < -0.08, u          # q / H = 0.5 / 5
    assert 0.0 < a["eta2"].mean() < 0.02
    assert np.isfinite(a["eta2"]).all()
