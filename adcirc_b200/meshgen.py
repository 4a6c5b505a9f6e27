"""Seeded synthetic meshes for the 2DDI hot path.

The benchmark meshes are synthetic by specification (no external dataset is
involved): a structured tidal channel (4,961 nodes), a small beach channel
with wetting/drying for parity tests, and a graded ~600k-node storm-surge
mesh.  Each generator returns a ``RawMesh``: node coordinates, bathymetric
depth (positive down, ADCIRC's DP), counter-clockwise triangles, one
elevation-specified (open) boundary and the land boundary segments with
their ADCIRC IBTYPE codes, listed counter-clockwise (domain on the left) as
in fort.14.
"""
from __future__ import annotations

import dataclasses
import numpy as np


@dataclasses.dataclass
class RawMesh:
    name: str
    x: np.ndarray          # (NP,) float64 [m]
    y: np.ndarray          # (NP,) float64 [m]
    dp: np.ndarray         # (NP,) float64, depth below datum [m]
    nm: np.ndarray         # (NE,3) int, 0-based node ids
    open_nodes: np.ndarray  # elevation boundary node ids (0-based), in order
    land_segments: list    # list of (ibtype, node id array (0-based))
    meta: dict
    # barrier segments, by segment index, per node: IBTYPE 3/13/23 (BARLANHT
    # crest heights [m above datum], BARLANCFSP); 4/24 (BARINHT, BARINCFSB,
    # BARINCFSP, the paired back-face nodes, 0-based); 5/25 those and
    # (PIPEHT, PIPECOEF, PIPEDIAM)
    barriers: dict = dataclasses.field(default_factory=dict)


def channel_mesh(nx: int = 121, ny: int = 41, lx: float = 60e3, ly: float = 20e3,
                 depth0: float = 20.0, depth1: float = 5.0) -> RawMesh:
    """Structured right-triangle channel: the 2DDI tidal channel case.

    Nodes are numbered column by column (x fastest along y); the open
    boundary is the x = 0 edge, the other three sides are mainland
    (IBTYPE 0).  Depth varies linearly in x from ``depth0`` to ``depth1``.
    """
    xs = np.linspace(0.0, lx, nx)
    ys = np.linspace(0.0, ly, ny)
    X, Y = np.meshgrid(xs, ys, indexing="ij")  # (nx, ny)
    x = X.ravel().astype(np.float64)
    y = Y.ravel().astype(np.float64)
    dp = depth0 + (depth1 - depth0) * (x / lx)

    def nid(i, j):
        return i * ny + j

    tris = []
    for i in range(nx - 1):
        for j in range(ny - 1):
            a, b, c, d = nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)
            tris.append((a, b, c))
            tris.append((a, c, d))
    nm = np.asarray(tris, dtype=np.int64)
    # open boundary: x = 0, from top (0, ly) down to (0, 0)
    open_nodes = np.array([nid(0, j) for j in range(ny - 1, -1, -1)], dtype=np.int64)
    # mainland: (0,0) -> (lx,0) -> (lx,ly) -> (0,ly), counter-clockwise
    land = [nid(i, 0) for i in range(nx)]
    land += [nid(nx - 1, j) for j in range(1, ny)]
    land += [nid(i, ny - 1) for i in range(nx - 2, -1, -1)]
    return RawMesh("channel", x, y, dp, nm, open_nodes,
                   [(0, np.asarray(land, dtype=np.int64))],
                   {"nx": nx, "ny": ny, "lx": lx, "ly": ly})


def levee_channel_mesh(crest: float, btype: int = 4, ib: int = 60, polder_depth: float = 0.0,
                       cfsb: float = 1.0, cfsp: float = 1.0, gap: float = 50.0, pipe=None,
                       **kw) -> RawMesh:
    """The channel with an internal barrier (IBTYPE `btype`, 4 or 24) along
    the column x = ib * dx: the column's inner nodes (all but the wall
    corners) are duplicated, the elements east of the column use the copies,
    and the two lines of nodes are the barrier's front (west) and back (east,
    `gap` metres further east) faces, paired in order, with crest height `crest` [m above datum] and
    discharge coefficients `cfsb` (subcritical) and `cfsp` (supercritical).
    East of the barrier the bed is flat at depth `polder_depth` (0: the
    datum, so the polder starts dry); the outer walls are one land segment
    as in `channel_mesh`.  For btype 5/25, `pipe` = (PIPEHT, PIPECOEF,
    PIPEDIAM) is the same pipe under every pair."""
    m = channel_mesh(**kw)
    nx, ny = m.meta["nx"], m.meta["ny"]
    nid = lambda i, j: i * ny + j
    npn = m.x.size
    front = np.array([nid(ib, j) for j in range(1, ny - 1)], dtype=np.int64)
    back = np.arange(npn, npn + front.size, dtype=np.int64)
    # the back face stands `gap` east of the front face: NEIGHB sorts a
    # node's neighbours by angle and cannot hold two at one place
    # (mesh.F:3223-3235), which a shared wall-corner node would have
    x = np.concatenate([m.x, m.x[front] + gap])
    y = np.concatenate([m.y, m.y[front]])
    dp = np.concatenate([m.dp, m.dp[front]])
    east = x > m.x[nid(ib, 0)]
    dp[east] = polder_depth
    dp[back] = polder_depth
    remap = np.arange(npn, dtype=np.int64)
    remap[front] = back
    nm = m.nm.copy()
    # elements of the columns east of the barrier line take the copies
    cx = m.x[m.nm].mean(axis=1)
    east_el = cx > m.x[nid(ib, 0)]
    nm[east_el] = remap[nm[east_el]]
    n = front.size
    bar = (np.full(n, float(crest)), np.full(n, float(cfsb)), np.full(n, float(cfsp)), back)
    if btype in (5, 25):
        bar += tuple(np.full(n, float(v)) for v in pipe)
    barriers = {1: bar}
    meta = dict(m.meta, barrier_column=ib)
    return RawMesh("levee_channel", x, y, dp, nm, m.open_nodes,
                   [m.land_segments[0], (int(btype), front)], meta, barriers)


def beach_mesh(nx: int = 41, ny: int = 13, lx: float = 4e3, ly: float = 1.2e3,
               depth0: float = 3.0, depth1: float = -1.5) -> RawMesh:
    """Small sloping-beach channel whose closed end rises above the datum.

    The tide floods and drains the upper beach, so every wet/dry branch
    of the path (D1, W1, DE1, D2, the slope limiter) is exercised on a
    mesh the oracle steps in well under a second.
    """
    m = channel_mesh(nx, ny, lx, ly, depth0, depth1)
    # a gentle cross-channel bump so fronts are not aligned with the grid
    m.dp = m.dp + 0.4 * np.sin(2.0 * np.pi * m.y / ly) * (m.x / lx)
    m.name = "beach"
    return m


def quarter_annulus_mesh(nr: int = 21, nth: int = 31, r1: float = 60.96e3, r2: float = 152.4e3,
                         h1: float = 3.048) -> RawMesh:
    """Quarter-annular harbour (Lynch and Gray's analytic test): r1 <= r <=
    r2, 0 <= theta <= 90 degrees, depth h1 (r / r1)^2 (3.048 m to 19.05 m),
    nr x nth nodes on a polar grid, each cell split along alternating
    diagonals.  The outer arc is the elevation boundary; the inner arc and
    the two radial sides are one mainland segment (IBTYPE 0)."""
    rs = np.linspace(r1, r2, nr)
    th = np.linspace(0.0, 0.5 * np.pi, nth)
    R, T = np.meshgrid(rs, th, indexing="ij")          # (nr, nth)
    x = (R * np.cos(T)).ravel()
    y = (R * np.sin(T)).ravel()
    dp = h1 * (R.ravel() / r1) ** 2

    def nid(i, j):
        return i * nth + j

    tris = []
    for i in range(nr - 1):
        for j in range(nth - 1):
            a, b, c, d = nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)
            if (i + j) % 2 == 0:
                tris += [(a, b, c), (a, c, d)]
            else:
                tris += [(a, b, d), (b, c, d)]
    nm = np.asarray(tris, np.int64)
    # outer arc, counter-clockwise (theta 0 -> 90 degrees)
    open_nodes = np.array([nid(nr - 1, j) for j in range(nth)], np.int64)
    # theta = 90 side inwards, inner arc back to theta = 0, theta = 0 side outwards
    land = [nid(i, nth - 1) for i in range(nr - 1, -1, -1)]
    land += [nid(0, j) for j in range(nth - 2, -1, -1)]
    land += [nid(i, 0) for i in range(1, nr)]
    return RawMesh("quarter_annulus", x, y, dp, nm, open_nodes,
                   [(0, np.asarray(land, np.int64))],
                   {"nr": nr, "nth": nth, "r1": r1, "r2": r2, "h1": h1,
                    "lx": r2, "ly": r2})


# --------------------------------------------------------------------------
# Graded storm-surge mesh
# --------------------------------------------------------------------------

def _coastline(rng, lx, y0, amp, nmodes=400, beta=1.35):
    k = np.arange(1, nmodes + 1, dtype=np.float64)
    a = amp * k ** (-beta) * rng.standard_normal(nmodes)
    ph = rng.uniform(0.0, 2.0 * np.pi, nmodes)

    def yc(x):
        x = np.asarray(x, dtype=np.float64)
        s = np.zeros_like(x)
        for kk, aa, pp in zip(k, a, ph):
            s += aa * np.sin(2.0 * np.pi * kk * x / lx + pp)
        return y0 + s
    return yc


def _grf(rng, lx, ly, dx, sigma, ell):
    nx = int(np.ceil(lx / dx)) + 1
    ny = int(np.ceil(ly / dx)) + 1
    w = rng.standard_normal((nx, ny))
    kx = np.fft.fftfreq(nx, d=dx) * 2 * np.pi
    ky = np.fft.rfftfreq(ny, d=dx) * 2 * np.pi
    KX, KY = np.meshgrid(kx, ky, indexing="ij")
    filt = np.exp(-0.25 * (KX ** 2 + KY ** 2) * ell ** 2)
    f = np.fft.irfft2(np.fft.rfft2(w) * filt, s=(nx, ny))
    f *= sigma / max(f.std(), 1e-30)

    def ev(x, y):
        fx = np.clip(x / dx, 0, nx - 1.000001)
        fy = np.clip(y / dx, 0, ny - 1.000001)
        i = fx.astype(np.int64)
        j = fy.astype(np.int64)
        tx = fx - i
        ty = fy - j
        return ((1 - tx) * (1 - ty) * f[i, j] + tx * (1 - ty) * f[i + 1, j]
                + (1 - tx) * ty * f[i, j + 1] + tx * ty * f[i + 1, j + 1])
    return ev


def _quadtree_leaves(lx, ly, h_fn, root):
    """Cells split until their size is below the target edge length."""
    nx0 = int(round(lx / root))
    ny0 = int(round(ly / root))
    I, J = np.meshgrid(np.arange(nx0), np.arange(ny0), indexing="ij")
    cx = (I.ravel() + 0.5) * root
    cy = (J.ravel() + 0.5) * root
    size = np.full(cx.shape, root)
    leaves = []
    while cx.size:
        h = h_fn(cx, cy, size)
        split = size > h
        leaves.append((cx[~split], cy[~split], size[~split]))
        cx, cy, size = cx[split], cy[split], size[split]
        if not cx.size:
            break
        q = size / 4.0
        cx = np.concatenate([cx - q, cx + q, cx - q, cx + q])
        cy = np.concatenate([cy - q, cy - q, cy + q, cy + q])
        size = np.concatenate([size, size, size, size]) / 2.0
    return (np.concatenate([l[0] for l in leaves]), np.concatenate([l[1] for l in leaves]),
            np.concatenate([l[2] for l in leaves]))


def _poisson_disk(px, py, h, fixed, beta, rng):
    """Thin candidate points to a Poisson-disk set: no two kept points closer
    than beta * min(h_i, h_j).  Conflicts come from each point's nearest
    candidates; a maximal independent set of the conflict graph is taken by
    random priorities (Luby's rounds), with the `fixed` points (boundary)
    always kept."""
    from scipy.spatial import cKDTree
    pts = np.column_stack([px, py])
    tree = cKDTree(pts)
    k = 12
    dist, idx = tree.query(pts, k=k)
    i = np.repeat(np.arange(px.size), k - 1)
    j = idx[:, 1:].ravel()
    d = dist[:, 1:].ravel()
    ok = j < px.size
    i, j, d = i[ok], j[ok], d[ok]
    conflict = d < beta * np.minimum(h[i], h[j])
    i, j = i[conflict], j[conflict]
    keep = i < j
    i, j = np.concatenate([i[keep], j[~keep]]), np.concatenate([j[keep], i[~keep]])
    pair = np.unique(i.astype(np.int64) * px.size + j)
    i, j = pair // px.size, pair % px.size
    prio = rng.random(px.size)
    prio[fixed] = 2.0 + prio[fixed]          # boundary points win every conflict
    state = np.zeros(px.size, np.int8)       # 0 undecided, 1 kept, -1 removed
    while True:
        live = (state[i] == 0) & (state[j] == 0)
        i, j = i[live], j[live]
        if i.size == 0:
            break
        # a point loses a round if some undecided neighbour has a higher priority
        lose = np.zeros(px.size, bool)
        lose[np.where(prio[i] < prio[j], i, j)] = True
        win = (state == 0) & ~lose
        state[win] = 1
        kill = np.concatenate([j[win[i]], i[win[j]]])
        state[kill[state[kill] == 0]] = -1
    state[state == 0] = 1
    return state == 1


def _edge_points(x0, y0, x1, y1, h_of):
    """Points along a domain edge at the local target spacing: the k-th
    point sits where the integral of 1/h along the edge reaches k (the
    endpoints included)."""
    L = float(np.hypot(x1 - x0, y1 - y0))
    t = np.linspace(0.0, L, int(L / 5.0) + 2)
    xs = x0 + (x1 - x0) * t / L
    ys = y0 + (y1 - y0) * t / L
    inv = 1.0 / h_of(xs, ys)
    n_int = np.concatenate([[0.0], np.cumsum(0.5 * (inv[1:] + inv[:-1]) * np.diff(t))])
    n = max(int(round(n_int[-1])), 1)
    tk = np.interp(np.linspace(0.0, n_int[-1], n + 1), n_int, t)
    return x0 + (x1 - x0) * tk / L, y0 + (y1 - y0) * tk / L


def surge_mesh(seed: int = 2024, target_nodes: int = 600_000, lx: float = 1000e3,
               ly: float = 800e3, h_min: float = 60.0, h_max: float = 20e3,
               coast_y: float = 640e3, coast_amp: float = 40e3,
               shelf_width: float = 100e3, shelf_depth: float = 30.0,
               ocean_depth: float = 4000.0, land_height: float = 6.0,
               grf_sigma: float = 2.0, grf_ell: float = 5e3,
               land_grading: float = 3.0, beta: float = 0.75, verbose: bool = False,
               alpha: float | None = None) -> RawMesh:
    """Graded storm-surge mesh (~600k nodes, ~1.2M triangles).

    Points: seeded Poisson-disk sampling whose spacing follows the target
    edge length h = min(h_max, h_min + alpha * d), d the distance to a
    seeded fractal coastline (the floodplain grades land_grading times
    faster): two uniform candidates per quadtree cell no larger than h are
    thinned so no two points are closer than beta * h; the domain edges
    carry points at spacing h; alpha is bisected so the node count meets the
    target.  Triangles: Delaunay (scipy).  Bathymetry: shelf profile
    (ocean_depth offshore, shelf break shelf_width offshore at shelf_depth,
    0 m at the coast, land rising to land_height) plus a Gaussian random
    field.  Open boundary: the south edge; the other sides are mainland
    (IBTYPE 0).
    """
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    yc = _coastline(rng, lx, coast_y, coast_amp)
    # coastline sampled once for fast distance evaluation (vertical proxy)
    xs = np.linspace(0, lx, 20001)
    ycs = yc(xs)

    def coast_at(x):
        return np.interp(x, xs, ycs)

    def make_h(alpha):
        def h_fn(cx, cy, size):
            s = coast_at(cx) - cy                  # > 0 offshore
            d = np.maximum(np.abs(s) - 0.75 * size, 0.0)   # nearest point of the cell
            a = np.where(s < 0, land_grading * alpha, alpha)
            return np.minimum(h_max, h_min + a * d)
        return h_fn

    def h_at(px, py):
        sd = coast_at(px) - py
        a = np.where(sd < 0, land_grading * alpha_cur[0], alpha_cur[0])
        return np.minimum(h_max, h_min + a * np.abs(sd))

    alpha_cur = [0.05]

    def candidates(alpha):
        alpha_cur[0] = alpha
        cx, cy, size = _quadtree_leaves(lx, ly, make_h(alpha), h_max)
        cx = np.repeat(cx, 2)
        cy = np.repeat(cy, 2)
        size = np.repeat(size, 2)
        px = cx + size * rng.uniform(-0.5, 0.5, cx.size)
        py = cy + size * rng.uniform(-0.5, 0.5, cy.size)
        return px, py

    # the thinned set keeps a stable fraction of the candidates: calibrate
    # it once, then bisect alpha on the candidate count
    given = alpha is not None
    lo, hi = 0.005, 0.5
    frac = 0.19
    mid = alpha
    for _ in range(0 if given else 40):
        mid = np.sqrt(lo * hi)
        cx, _, _ = _quadtree_leaves(lx, ly, make_h(mid), h_max)
        if 2 * cx.size * frac > target_nodes:
            lo = mid
        else:
            hi = mid
        if abs(2 * cx.size * frac - target_nodes) < 0.005 * target_nodes:
            break
    alpha = mid
    for attempt in range(3):
        px, py = candidates(alpha)
        hb = h_at(px, py)
        inside = ((px > 0.5 * hb) & (px < lx - 0.5 * hb) & (py > 0.5 * hb) & (py < ly - 0.5 * hb))
        px, py, hb = px[inside], py[inside], hb[inside]
        bx, by = [], []
        for (x0, y0, x1, y1) in [(0, 0, lx, 0), (lx, 0, lx, ly), (lx, ly, 0, ly), (0, ly, 0, 0)]:
            ex, ey = _edge_points(x0, y0, x1, y1, h_at)
            bx.append(ex[:-1])
            by.append(ey[:-1])
        bx = np.concatenate(bx)
        by = np.concatenate(by)
        nb = bx.size
        ax = np.concatenate([bx, px])
        ay = np.concatenate([by, py])
        fixed = np.zeros(ax.size, bool)
        fixed[:nb] = True
        kept = _poisson_disk(ax, ay, h_at(ax, ay), fixed, beta, rng)
        n_kept = int(kept.sum())
        if verbose:
            print(f"surge_mesh: alpha {alpha:.5f} candidates {ax.size} kept {n_kept}")
        if given or abs(n_kept - target_nodes) < 0.015 * target_nodes:
            break
        # the node count scales about as alpha^-0.95 for these gradings
        alpha *= (n_kept / target_nodes) ** (1.0 / 0.95)
    x = ax[kept]
    y = ay[kept]
    # boundary points bulge outward by a tiny convex offset so that every
    # one is a hull vertex of the triangulation
    onb = np.zeros(x.size, bool)
    onb[:nb] = True
    for (cond, nx_, ny_, L) in [(np.abs(y) < 1e-6, 0.0, -1.0, lx), (np.abs(x - lx) < 1e-6, 1.0, 0.0, ly),
                                (np.abs(y - ly) < 1e-6, 0.0, 1.0, lx), (np.abs(x) < 1e-6, -1.0, 0.0, ly)]:
        m = onb & cond
        sfrac = (x[m] / L) if nx_ == 0.0 else (y[m] / L)
        bulge = 1e-6 * L * sfrac * (1 - sfrac) * 4.0
        x[m] = x[m] + nx_ * bulge
        y[m] = y[m] + ny_ * bulge
    tri = Delaunay(np.column_stack([x, y]))
    nm = tri.simplices.astype(np.int64)
    # orient counter-clockwise
    x1, y1 = x[nm[:, 0]], y[nm[:, 0]]
    x2, y2 = x[nm[:, 1]], y[nm[:, 1]]
    x3, y3 = x[nm[:, 2]], y[nm[:, 2]]
    a2 = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1)
    flip = a2 < 0
    nm[flip, 1], nm[flip, 2] = nm[flip, 2].copy(), nm[flip, 1].copy()
    # drop degenerate triangles (zero area) if any
    keep = np.abs(a2) > 1e-6 * np.median(np.abs(a2))
    nm = nm[keep]
    used = np.zeros(x.size, bool)
    used[nm.ravel()] = True
    if not used.all():
        remap = -np.ones(x.size, np.int64)
        remap[used] = np.arange(used.sum())
        x, y = x[used], y[used]
        nm = remap[nm]
        nb = int(used[:nb].sum())
    # renumber for memory locality: nodes along a Hilbert curve, elements by
    # their lowest node
    key = _hilbert_key(x, y, lx, ly)
    perm = np.argsort(key, kind="stable")
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    x, y = x[perm], y[perm]
    nm = inv[nm]
    ekey = np.lexsort((nm.max(axis=1), nm.min(axis=1)))
    nm = nm[ekey]
    # bathymetry
    grf = _grf(rng, lx, ly, 1250.0, grf_sigma, grf_ell)
    s = coast_at(x) - y  # > 0 offshore
    shelf = shelf_depth * np.sqrt(np.clip(s / shelf_width, 0.0, 1.0))
    slope = 0.5 * (1 + np.tanh((s - shelf_width - 25e3) / 12e3))
    depth = shelf + (ocean_depth - shelf_depth) * slope * (s > shelf_width)
    land = s < 0
    depth = np.where(land, -land_height * np.clip(-s / 20e3, 0.0, 1.0), depth)
    depth = depth + grf(x, y) * np.clip(1.0 - s / (2 * shelf_width), 0.0, 1.0)
    depth = np.clip(depth, -land_height, ocean_depth)
    # boundary node lists from hull ordering (counter-clockwise)
    bnd = _hull_loop(nm, x.size)
    # start the loop at the south-west corner
    corner = int(np.argmin(x[bnd] + y[bnd]))
    bnd = np.roll(bnd, -corner)
    # counter-clockwise: south edge first (increasing x)
    if x[bnd[1]] < x[bnd[0]]:
        bnd = np.concatenate([bnd[:1], bnd[1:][::-1]])
    tol = 1.0
    south = np.abs(y[bnd]) < tol + 1e-6 * lx
    # open boundary: the south edge, listed as in fort.14 from east to west
    # (so that the land boundary continues counter-clockwise from it)
    i_end = int(np.argmax(~south[1:])) + 1  # first non-south after start
    open_ccw = bnd[:i_end]                   # west -> east along the south edge
    open_nodes = open_ccw[::-1]
    land_nodes = np.concatenate([bnd[i_end - 1:], bnd[:1]])  # SE corner -> ... -> SW corner
    meta = {"seed": seed, "alpha": float(alpha), "coast_y": coast_y, "lx": lx, "ly": ly}
    rm = RawMesh("surge", x.astype(np.float64), y.astype(np.float64), depth.astype(np.float64),
                 nm, open_nodes.astype(np.int64), [(0, land_nodes.astype(np.int64))], meta)
    rm.meta["coast_fn"] = coast_at
    return rm


def _hilbert_key(x, y, lx, ly, order=16):
    n = 1 << order
    xi = np.clip((x / lx * (n - 1)).astype(np.int64), 0, n - 1)
    yi = np.clip((y / ly * (n - 1)).astype(np.int64), 0, n - 1)
    d = np.zeros_like(xi)
    s = n >> 1
    while s > 0:
        rx = ((xi & s) > 0).astype(np.int64)
        ry = ((yi & s) > 0).astype(np.int64)
        d += s * s * ((3 * rx) ^ ry)
        # rotate
        mask = ry == 0
        flip = mask & (rx == 1)
        xi = np.where(flip, s - 1 - xi, xi)
        yi = np.where(flip, s - 1 - yi, yi)
        xi2 = np.where(mask, yi, xi)
        yi2 = np.where(mask, xi, yi)
        xi, yi = xi2, yi2
        s >>= 1
    return d


def _hull_loop(nm, npts):
    """Boundary edges (used by exactly one triangle) chained into a loop,
    oriented counter-clockwise (interior on the left)."""
    e = np.concatenate([nm[:, [0, 1]], nm[:, [1, 2]], nm[:, [2, 0]]])
    key = np.minimum(e[:, 0], e[:, 1]) * npts + np.maximum(e[:, 0], e[:, 1])
    uniq, cnt = np.unique(key, return_counts=True)
    bkeys = set(uniq[cnt == 1].tolist())
    nxt = {}
    for a, b, k in zip(e[:, 0], e[:, 1], key):
        if int(k) in bkeys:
            nxt[int(a)] = int(b)  # ccw triangles: boundary edge a->b has interior on the left
    start = next(iter(nxt))
    loop = [start]
    cur = nxt[start]
    while cur != start:
        loop.append(cur)
        cur = nxt[cur]
        if len(loop) > len(nxt) + 1:
            raise RuntimeError("boundary is not a single loop")
    return np.asarray(loop, dtype=np.int64)
