"""Seeded swept-wing cloud in the reference's input layout.

A half wing with a NACA 0012 section (closed trailing edge), semispan 1,
taper 0.56 and a 30 deg leading-edge sweep, spanwise along +z from the
symmetry plane z = 0.  Its surface carries 400 chordwise x 120 spanwise wall
points (status 1), and 300 more close the tip (a flat tip face, normal +z).  Volume points fill the half box [-10, 10]^2 x [0, 10]
with a density proportional to exp(-d / 0.3) in the distance d to the
wing's surface plus a uniform floor, drawn by rejection sampling over a
grid of cells refined near the wing.  Points within about one local spacing
of the box faces or of the symmetry plane are outer points (status 2), so
the symmetry plane is a far-field boundary; all other volume points are
interior (status 0, global frame).

The reference reads clouds from a file and ships none; this generator is
the project's, seeded and built only from host-independent arithmetic (IEEE
+, -, *, /, sqrt and the C library's scalar transcendentals), like
cloud.shell_cloud, except that the volume sampling uses numpy's vectorised
exp for its acceptance tests (a cloud regenerated on another host may
differ in rare accepted points).  The cloud is stored wall points first,
then the interior points along a Morton curve, then the outer points.

Connectivity is the 26 nearest neighbours, cut to the 22 nearest where a
split list would otherwise exceed the reference's 22 entries of storage
(data_structure.f90:83-88): at every wall and outer point (their z list is
the whole neighbourhood) and at interior points with a lopsided half, so no
list overflows into another point's storage.  A last pass checks every
interior and wall point's six least-squares lists as the reference builds
them (generate_connectivity.f90:38-246): volume points whose lists have
fewer than three members or a (near-)singular 3x3 system are removed (a
wall point in that state gets two volume points just off the surface beside
it) and the neighbours recomputed; what remains after the last round is
made an outer point.
"""
from __future__ import annotations

import math

import numpy as np

from .cloud import (MAX_CONN, STATUS_INTERIOR, STATUS_OUTER, STATUS_WALL, PointCloud, _boundary_frames,
                    _knn_connectivity, _rows_norm)

THICKNESS = 0.12
SEMISPAN = 1.0
ROOT_CHORD = 1.0
TAPER = 0.56
SWEEP_DEG = 30.0
BOX = 10.0
DECAY = 0.3


def _tan_sweep() -> float:
    a = SWEEP_DEG * (4.0 * math.atan(1.0)) / 180.0
    return math.sin(a) / math.cos(a)


def half_thickness(xi: np.ndarray) -> np.ndarray:
    """NACA 00xx half thickness over the chord, closed trailing edge (the
    published 4-digit formula with the -0.1036 x^4 term)."""
    xi = np.clip(xi, 0.0, 1.0)
    return 5.0 * THICKNESS * (0.2969 * np.sqrt(xi) - 0.1260 * xi - 0.3516 * xi * xi
                              + 0.2843 * xi * xi * xi - 0.1036 * xi * xi * xi * xi)


def half_thickness_slope(xi: np.ndarray) -> np.ndarray:
    xi = np.clip(xi, 1e-12, 1.0)
    return 5.0 * THICKNESS * (0.5 * 0.2969 / np.sqrt(xi) - 0.1260 - 2.0 * 0.3516 * xi
                              + 3.0 * 0.2843 * xi * xi - 4.0 * 0.1036 * xi * xi * xi)


def chord(z: np.ndarray) -> np.ndarray:
    return ROOT_CHORD * (1.0 - (1.0 - TAPER) * z / SEMISPAN)


def leading_edge_x(z: np.ndarray) -> np.ndarray:
    return z * _tan_sweep()


def surface(xi: np.ndarray, z: np.ndarray, side: np.ndarray):
    """Points, outward unit normals and area elements |dP/dxi x dP/dz| of the
    surface at chord fraction xi, span z, side +1 (upper) or -1 (lower)."""
    c = chord(z)
    dc = -ROOT_CHORD * (1.0 - TAPER) / SEMISPAN
    t = half_thickness(xi)
    tp = half_thickness_slope(xi)
    ts = _tan_sweep()
    p = np.stack([leading_edge_x(z) + xi * c, side * c * t, z], axis=1)
    # a = dP/dxi = (c, s c t', 0); b = dP/dz = (tan L + xi c', s c' t, 1)
    ax, ay = c, side * c * tp
    bx, by = ts + xi * dc, side * dc * t
    nx = ay
    ny = -ax
    nz = ax * by - ay * bx
    n = np.stack([nx, ny, nz], axis=1)
    area = _rows_norm(n)
    n = n / area[:, None]
    flip = np.sign(n[:, 1]) != side
    n[flip] = -n[flip]
    return p, n, area


def inside_wing(pts: np.ndarray) -> np.ndarray:
    """True where a point lies inside the wing (or on its surface)."""
    x, y, z = pts[:, 0], pts[:, 1], pts[:, 2]
    inz = (z >= 0.0) & (z <= SEMISPAN)
    zc = np.clip(z, 0.0, SEMISPAN)
    c = chord(zc)
    xi = (x - leading_edge_x(zc)) / c
    inx = (xi >= 0.0) & (xi <= 1.0)
    return inz & inx & (np.abs(y) <= c * half_thickness(xi))


def wall_grid(nc: int = 400, ns: int = 120):
    """Wall points of the surface grid: nc/2 chordwise stations per side
    (xi = s/2 + (1 - cos(pi s / 2))/2, finer toward the leading edge, cell
    centred) x ns spanwise stations
    (cell centred).  Returns points, normals, areas, and the parameter
    cells (xi_lo, xi_hi, z_lo, z_hi, side) they stand for."""
    half = nc // 2
    pi = 4.0 * math.atan(1.0)
    def xi_of(s):   # half uniform, half clustered toward the leading edge
        return 0.5 * s + 0.5 * (1.0 - math.cos(0.5 * pi * s))
    edges = np.array([xi_of(i / half) for i in range(half + 1)])
    xi_c = np.array([xi_of((i + 0.5) / half) for i in range(half)])
    z_edges = SEMISPAN * np.arange(ns + 1, dtype=np.float64) / ns
    z_c = SEMISPAN * (np.arange(ns, dtype=np.float64) + 0.5) / ns
    xi = np.concatenate([np.tile(xi_c, ns), np.tile(xi_c, ns)])
    dxi = np.concatenate([np.tile(edges[1:] - edges[:-1], ns)] * 2)
    z = np.concatenate([np.repeat(z_c, half), np.repeat(z_c, half)])
    side = np.concatenate([np.ones(half * ns), -np.ones(half * ns)])
    p, n, da = surface(xi, z, side)
    area = da * dxi * (SEMISPAN / ns)
    cells = (np.concatenate([np.tile(edges[:-1], ns)] * 2), np.concatenate([np.tile(edges[1:], ns)] * 2),
             np.concatenate([np.repeat(z_edges[:-1], half)] * 2), np.concatenate([np.repeat(z_edges[1:], half)] * 2),
             side)
    return p, n, area, cells


def tip_cap(nc: int = 400):
    """Wall points closing the tip: the section face at z = semispan, nc/4
    chordwise stations (the surface grid's leading-edge clustering) x three
    rows across the thickness, normal +z; returns points, normals, areas."""
    m = max(4, nc // 4)
    pi = 4.0 * math.atan(1.0)
    xi = np.array([0.5 * (i + 0.5) / m + 0.5 * (1.0 - math.cos(0.5 * pi * (i + 0.5) / m)) for i in range(m)])
    edges = np.array([0.5 * i / m + 0.5 * (1.0 - math.cos(0.5 * pi * i / m)) for i in range(m + 1)])
    c = chord(np.array([SEMISPAN]))[0]
    t = half_thickness(xi) * c
    rows, areas = [], []
    for f in (-0.5, 0.0, 0.5):
        rows.append(np.stack([leading_edge_x(np.full(m, SEMISPAN)) + xi * c, f * t, np.full(m, SEMISPAN)], axis=1))
        areas.append((edges[1:] - edges[:-1]) * c * (2.0 * t) / 3.0)
    p = np.concatenate(rows)
    n = np.zeros_like(p)
    n[:, 2] = 1.0
    return p, n, np.concatenate(areas)


def _surface_tree(nc: int = 1200, ns: int = 360):
    """k-d tree of a dense sampling of the whole surface (both sides and the
    tip face), for distances from the wing."""
    from scipy.spatial import cKDTree
    p, _, _, _ = wall_grid(nc, ns)
    # tip face: the section at z = semispan
    m = 200
    xi = (np.arange(m, dtype=np.float64) + 0.5) / m
    c = chord(np.array([SEMISPAN]))[0]
    t = half_thickness(xi) * c
    rows = []
    for j in range(9):
        f = -1.0 + 2.0 * j / 8.0
        rows.append(np.stack([leading_edge_x(np.full(m, SEMISPAN)) + xi * c, f * t, np.full(m, SEMISPAN)],
                             axis=1))
    return cKDTree(np.concatenate([p] + rows))


def _layer_points(rng, tree, amp: float) -> np.ndarray:
    """Poisson points of density amp * exp(-d / DECAY) in the half box, by
    rejection from cells whose size adapts to the density's variation."""
    lo = np.array([-BOX, -BOX, 0.0])
    size = 2.5
    counts = (np.array([2 * BOX, 2 * BOX, BOX]) / size).astype(int)
    g = np.stack(np.meshgrid(*[np.arange(k) for k in counts], indexing="ij"), axis=-1).reshape(-1, 3)
    centres = lo + (g + 0.5) * size
    half = np.full(len(centres), 0.5 * size)
    leaves_c, leaves_h, leaves_b = [], [], []
    while len(centres):
        d, _ = tree.query(centres, workers=-1)
        r = np.sqrt(3.0) * half
        dmin = np.maximum(0.0, d - r)
        hi = np.exp(-dmin / DECAY)
        low = np.exp(-(d + r) / DECAY)
        split = (hi > 1.5 * low) & (half > 0.02) & (hi * amp * (2 * half) ** 3 > 0.5)
        keep = ~split & (hi * amp * (2 * half) ** 3 > 1e-3)
        leaves_c.append(centres[keep])
        leaves_h.append(half[keep])
        leaves_b.append(amp * hi[keep])
        cs, hs = centres[split], half[split] * 0.5
        offs = np.array([[sx, sy, sz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)], dtype=np.float64)
        centres = (cs[:, None, :] + offs[None, :, :] * hs[:, None, None]).reshape(-1, 3)
        half = np.repeat(hs, 8)
    cc, hh, bb = np.concatenate(leaves_c), np.concatenate(leaves_h), np.concatenate(leaves_b)
    vol = (2.0 * hh) ** 3
    k = rng.poisson(bb * vol)
    idx = np.repeat(np.arange(len(cc)), k)
    u = rng.uniform(-1.0, 1.0, size=(len(idx), 3))
    pts = cc[idx] + u * hh[idx, None]
    d, _ = tree.query(pts, workers=-1)
    accept = rng.uniform(0.0, 1.0, size=len(pts)) * bb[idx] < amp * np.exp(-d / DECAY)
    return pts[accept], d[accept]


def _morton_keys(pts: np.ndarray) -> np.ndarray:
    lo = pts.min(axis=0)
    span = np.maximum(pts.max(axis=0) - lo, 1e-300)
    q = np.clip(((pts - lo) / span * 2097151.0), 0, 2097151).astype(np.uint64)

    def spread(v):
        v = v & np.uint64(0x1fffff)
        v = (v | (v << np.uint64(32))) & np.uint64(0x1f00000000ffff)
        v = (v | (v << np.uint64(16))) & np.uint64(0x1f0000ff0000ff)
        v = (v | (v << np.uint64(8))) & np.uint64(0x100f00f00f00f00f)
        v = (v | (v << np.uint64(4))) & np.uint64(0x10c30c30c30c30c3)
        v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
        return v
    return spread(q[:, 0]) | (spread(q[:, 1]) << np.uint64(1)) | (spread(q[:, 2]) << np.uint64(2))


def _list_check(pts, cls, tan1, tan2, nor, nbhs, conn, lo, hi, cap=22):
    """Points of [lo, hi) whose split lists (generate_connectivity.f90:38-246)
    have fewer than three members or a 3x3 least-squares system singular to
    1e-9 relative; and the points with a list longer than the reference's
    `cap` entries of storage (data_structure.f90:83-88)."""
    k = conn[lo:hi, :nbhs.max()] - 1
    valid = np.arange(k.shape[1])[None, :] < nbhs[lo:hi, None]
    k = np.where(valid, k, 0)
    d = pts[k] - pts[lo:hi, None, :]
    t1, t2, nn = tan1[lo:hi, None, :], tan2[lo:hi, None, :], nor[lo:hi, None, :]
    ds = (d * t1).sum(axis=2)
    dt = (d * t2).sum(axis=2)
    dn = (d * nn).sum(axis=2)
    wall = (cls[lo:hi] == STATUS_WALL)[:, None]
    lists = [valid & (ds <= 0.0), valid & np.where(wall, ds >= 0.0, ds > 0.0),
             valid & (dt <= 0.0), valid & np.where(wall, dt >= 0.0, dt > 0.0),
             valid & ~wall & (dn <= 0.0), valid & np.where(wall, True, dn > 0.0)]
    bad = np.zeros(hi - lo, dtype=bool)
    over = np.zeros(hi - lo, dtype=bool)
    for li, m in enumerate(lists):
        if li == 4:
            m = m & ~wall   # a wall point has no z+ list
        cnt = m.sum(axis=1)
        over |= cnt > cap
        w = m.astype(np.float64)
        xx, yy, zz = (w * ds * ds).sum(1), (w * dt * dt).sum(1), (w * dn * dn).sum(1)
        xy, yz, zx = (w * ds * dt).sum(1), (w * dt * dn).sum(1), (w * dn * ds).sum(1)
        det = xx * (yy * zz - yz * yz) - xy * (xy * zz - yz * zx) + zx * (xy * yz - yy * zx)
        tr = (xx + yy + zz) / 3.0
        need = ~wall[:, 0] if li == 4 else np.ones(hi - lo, dtype=bool)
        bad |= need & ((cnt < 3) | (det <= 1e-9 * tr * tr * tr))
    return bad, over


def _deep_inside(pts: np.ndarray, frac: float = 0.7) -> np.ndarray:
    """Inside the wing by more than (1 - frac) of the local half thickness:
    the chord between two points of one side of the surface dips inside it
    only by its sag, a segment through the section crosses this core."""
    x, y, z = pts[:, 0], pts[:, 1], pts[:, 2]
    inz = (z >= 0.0) & (z < SEMISPAN * (1.0 - 1e-9))   # the tip face itself is not inside
    zc = np.clip(z, 0.0, SEMISPAN)
    c = chord(zc)
    xi = (x - leading_edge_x(zc)) / c
    return inz & (xi > 0.0) & (xi < 1.0) & (np.abs(y) < frac * c * half_thickness(xi))


def _visible_knn(pts: np.ndarray, k: int, tree, extra: int = 16, nwall: int = 0):
    """The k nearest neighbours of every point that it sees: a candidate is
    dropped when the segment to it passes through the wing (sampled at seven
    interior points), so no stencil couples the two sides of the thin
    trailing edge through the body; the first `nwall` points (walls) take at
    most k - k//3 wall points.  Points near the wing may keep fewer than k.  Returns nbhs, conn (1-based, zero padded) and min_dist, like
    cloud._knn_connectivity."""
    from scipy.spatial import cKDTree
    n = pts.shape[0]
    m = k + extra
    dist, idx = cKDTree(pts).query(pts, k=m + 1, workers=-1)
    if not np.all(idx[:, 0] == np.arange(n)):
        raise ValueError("duplicate points in generated cloud")
    idx, dist = idx[:, 1:], dist[:, 1:]
    ok = np.ones((n, m), dtype=bool)
    dw, _ = tree.query(pts, workers=-1)
    near = np.nonzero(dw < dist[:, -1])[0]      # only these can see through the wing
    step = 50_000
    for a in range(0, len(near), step):
        rows = near[a:a + step]
        p0 = pts[rows][:, None, :]
        d = pts[idx[rows]] - p0
        blocked = np.zeros((len(rows), m), dtype=bool)
        for f in (0.125, 0.25, 0.375, 0.5, 0.625, 0.75, 0.875):
            q = (p0 + f * d).reshape(-1, 3)
            blocked |= _deep_inside(q).reshape(len(rows), m)
        ok[rows] = ~blocked
    # the first k visible candidates, in distance order; a wall point takes
    # at most k - k//3 wall neighbours, so its lists always reach off the
    # surface (a stencil of surface points alone leaves the derivative along
    # the normal nearly undetermined)
    if nwall:
        is_wall_cand = idx < nwall
        cap_w = k - k // 3
        wrank = np.cumsum(ok & is_wall_cand, axis=1)
        ok[:nwall] &= ~(is_wall_cand[:nwall] & (wrank[:nwall] > cap_w))
    rank = np.cumsum(ok, axis=1)
    take = ok & (rank <= k)
    nbhs = take.sum(axis=1).astype(np.int32)
    conn = np.zeros((n, MAX_CONN), dtype=np.int32)
    order = np.argsort(~take, axis=1, kind="stable")[:, :k]
    sel = np.take_along_axis(idx, order, axis=1) + 1
    keep = np.arange(k)[None, :] < nbhs[:, None]
    conn[:, :k] = np.where(keep, sel, 0)
    kk = conn[:, 0] - 1
    dx = pts[kk] - pts
    md = np.sqrt(dx[:, 0] * dx[:, 0] + dx[:, 1] * dx[:, 1] + dx[:, 2] * dx[:, 2])
    return nbhs, conn, md


def _ghosts(pts: np.ndarray, h: np.ndarray, reach: float):
    """Outer points mirroring every point within reach * h of a face of the
    half box (the symmetry plane z = 0 included) to the other side of that
    face, with the face's outward normal.  Points within h / 4 of the face
    are not mirrored: their image would nearly coincide with them."""
    planes = [(0, -BOX, -1.0), (0, BOX, 1.0), (1, -BOX, -1.0), (1, BOX, 1.0), (2, 0.0, -1.0), (2, BOX, 1.0)]
    out, nors = [], []
    for axis, at, sgn in planes:
        dist = (at - pts[:, axis]) * sgn
        sel = (dist < reach * h) & (dist > 0.25 * h)
        g = pts[sel].copy()
        g[:, axis] = 2.0 * at - g[:, axis]
        nv = np.zeros((len(g), 3))
        nv[:, axis] = sgn
        out.append(g)
        nors.append(nv)
    return np.concatenate(out), np.concatenate(nors)


def swept_wing(points: int = 4_200_000, seed: int = 3001, k: int = 26, nc: int = 400, ns: int = 120,
               floor: float = 150.0, name: str = "wing-4.2M", rounds: int = 6) -> PointCloud:
    """The seeded swept-wing cloud (module docstring).  `points` is the
    target total; smaller clouds of the same construction for tests take a
    coarser wall grid (nc x ns)."""
    from scipy.spatial import cKDTree
    rng = np.random.Generator(np.random.PCG64(seed))
    pw, nw, aw, _ = wall_grid(nc, ns)
    pc, ncap, acap = tip_cap(nc)
    pw, nw, aw = np.concatenate([pw, pc]), np.concatenate([nw, ncap]), np.concatenate([aw, acap])
    tree = _surface_tree(max(nc, 240), max(ns, 72))
    box_vol = (2 * BOX) * (2 * BOX) * BOX
    n_floor = min(floor * box_vol, 0.2 * points)
    n_layer = max(0.0, 0.972 * points - len(pw) - n_floor)
    # the layer's amplitude: a first draw at a guessed amplitude, then thinned
    # (the integral of exp(-d / 0.3) over the half box around this wing is
    # about 1.65)
    amp = 1.15 * n_layer / 1.65
    while True:
        lay, dl = _layer_points(rng, tree, amp)
        if len(lay) >= n_layer:
            break
        amp *= 1.5 * n_layer / max(len(lay), 1)
    keep = rng.uniform(0.0, 1.0, size=len(lay)) < n_layer / len(lay)
    lay, dl = lay[keep], dl[keep]
    m = rng.poisson(n_floor)
    flo = rng.uniform(0.0, 1.0, size=(m, 3)) * np.array([2 * BOX, 2 * BOX, BOX]) + np.array([-BOX, -BOX, 0.0])
    dfl, _ = tree.query(flo, workers=-1)
    vol = np.concatenate([lay, flo])
    dv = np.concatenate([dl, dfl])
    # nothing inside the wing, and no volume point nearer the surface than a
    # fraction of the wall spacing
    ok = ~inside_wing(vol) & (dv > 0.0025 * ROOT_CHORD * 400.0 / nc)
    vol = vol[ok]
    vol = vol[np.argsort(_morton_keys(vol), kind="stable")]
    nwall = len(pw)
    for rnd in range(rounds):
        last = rnd == rounds - 1
        inner = np.concatenate([pw, vol])
        dist, _ = cKDTree(inner).query(inner, k=7, workers=-1)
        gp, gn = _ghosts(inner, dist[:, 6], 2.5)
        gp_order = np.argsort(_morton_keys(gp), kind="stable")
        gp, gn = gp[gp_order], gn[gp_order]
        pts = np.concatenate([inner, gp])
        n = len(pts)
        status = np.full(n, STATUS_INTERIOR, dtype=np.int32)
        status[:nwall] = STATUS_WALL
        status[len(inner):] = STATUS_OUTER
        nor = np.zeros((n, 3))
        nor[:, 2] = 1.0
        tan1 = np.zeros((n, 3))
        tan1[:, 0] = 1.0
        tan2 = np.zeros((n, 3))
        tan2[:, 1] = 1.0
        bnor = np.concatenate([nw, gn])
        bidx = np.concatenate([np.arange(nwall), np.arange(len(inner), n)])
        t1b, t2b = _boundary_frames(bnor)
        tan1[bidx], tan2[bidx], nor[bidx] = t1b, t2b, bnor
        nbhs, conn, md = _visible_knn(pts, k, tree, extra=24, nwall=nwall)
        # no list may exceed the reference's 22 entries of storage (an
        # overflowing list spills into the next point's column): wall and
        # outer points, whose z list is their whole neighbourhood, and
        # interior points with a lopsided half keep their 22 nearest
        cap = 22
        short = status != STATUS_INTERIOR
        step = 200_000
        for a in range(0, n, step):
            b = min(n, a + step)
            short[a:b] |= _list_check(pts, status, tan1, tan2, nor, nbhs, conn, a, b, cap)[1]
        nbhs[short] = np.minimum(nbhs[short], cap)
        conn[np.arange(MAX_CONN)[None, :] >= nbhs[:, None]] = 0
        bad = np.zeros(n, dtype=bool)
        for a in range(0, len(inner), step):
            b = min(len(inner), a + step)
            bad[a:b] = _list_check(pts, status, tan1, tan2, nor, nbhs, conn, a, b, cap)[0]
        drop = bad[nwall:len(inner)]
        if not bad[:len(inner)].any():
            break
        if last:
            # what is left after the last round becomes a far-field (outer)
            # point: it is not swept and its own lists are not used
            status[nwall:len(inner)][drop] = STATUS_OUTER
            break
        # a wall point whose lists are one-sided gets two volume points just
        # off the surface, one to either side along its tan2 direction
        wb = np.nonzero(bad[:nwall])[0]
        if len(wb):
            hw = dist[wb, 6]
            add = [pw[wb] + 0.5 * hw[:, None] * nw[wb] + sgn * 0.5 * hw[:, None] * tan2[wb]
                   + 0.05 * hw[:, None] * rng.uniform(-1.0, 1.0, size=(len(wb), 3)) for sgn in (-1.0, 1.0)]
            vol = np.concatenate([vol[~drop]] + add)
        else:
            vol = vol[~drop]
    area = np.zeros(n)
    area[:nwall] = aw
    c = PointCloud(status=status, x=np.ascontiguousarray(pts[:, 0]), y=np.ascontiguousarray(pts[:, 1]),
                   z=np.ascontiguousarray(pts[:, 2]), tan1=tan1, tan2=tan2, nor=nor, nbhs=nbhs, conn=conn,
                   min_dist=md, name=name, wall_area=float(aw.sum()),
                   ref_area=SEMISPAN * 0.5 * (1.0 + TAPER) * ROOT_CHORD, wall_areas=area)
    c.bad_lists = int(bad[:nwall].sum() + (bad[nwall:] & (status[nwall:] != STATUS_OUTER)).sum())
    c.bad_wall_lists = int(bad[:nwall].sum())
    return c
