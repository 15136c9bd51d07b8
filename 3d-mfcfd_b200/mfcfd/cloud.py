"""Seeded synthetic point clouds in the reference's input layout.

The reference reads its point cloud from a text file whose records are
``idx status x y z tan1(3) tan2(3) nor(3) nbhs conn(1..nbhs) min_dist``
(point_preprocessor.f90:30-36) into the arrays of ``type points``
(data_structure.f90:7-22).  No such file ships with the reference, so the
clouds here are generated: concentric shells around a sphere (or an
ellipsoid) with the body surface as the wall (status 1), the last shell as
the outer boundary (status 2) and everything else interior (status 0).

Arrays use the reference's memory order: a Fortran ``(3, N)`` array is a
C-order ``(N, 3)`` numpy array, ``conn(27, N)`` is ``(N, 27)`` int32 holding
1-based indices padded with 0, ``prim(5, N)`` is ``(N, 5)``.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

MAX_CONN = 27          # data_structure.f90:80  conn(27, max_points)

STATUS_INTERIOR = 0
STATUS_WALL = 1
STATUS_OUTER = 2
STATUS_SUPERSONIC_INLET = 5
STATUS_SUPERSONIC_OUTLET = 6


@dataclasses.dataclass
class PointCloud:
    """Geometry and connectivity of one cloud (reference ``type points``)."""
    status: np.ndarray      # (N,) int32
    x: np.ndarray           # (N,) float64
    y: np.ndarray
    z: np.ndarray
    tan1: np.ndarray        # (N, 3) float64 == Fortran tan1(3, N)
    tan2: np.ndarray
    nor: np.ndarray
    nbhs: np.ndarray        # (N,) int32
    conn: np.ndarray        # (N, 27) int32, 1-based, zero padded
    min_dist: np.ndarray    # (N,) float64
    name: str = "cloud"
    wall_area: float = 0.0  # surface area of the body (for force integration)
    ref_area: float = 0.0   # projected reference area for CL/CD
    wall_areas: np.ndarray | None = None   # (N,) per-point surface areas, or None: wall_area split evenly

    @property
    def n(self) -> int:
        return int(self.status.shape[0])

    def counts(self) -> dict:
        s = self.status
        return {"wall": int((s == STATUS_WALL).sum()),
                "outer": int((s == STATUS_OUTER).sum()),
                "interior": int((s == STATUS_INTERIOR).sum()),
                "supersonic_inlet": int((s == STATUS_SUPERSONIC_INLET).sum()),
                "supersonic_outlet": int((s == STATUS_SUPERSONIC_OUTLET).sum())}


def freestream(mach: float, aoa_deg: float):
    """Freestream primitive state as parameter.f90:19-33 defines it.

    ``theta = aoa*pi/180`` with ``pi = 4*atan(1)``; ``u1 = Mach*cos(theta)``,
    ``u2 = Mach*sin(theta)``, ``u3 = 0``, ``rho = 1``, ``p = 1/1.4``.
    """
    pi = 4.0 * math.atan(1.0)
    theta = aoa_deg * pi / 180.0
    return (1.0, mach * math.cos(theta), mach * math.sin(theta), 0.0, 1.0 / 1.4)


def freestream_prim(n: int, mach: float, aoa_deg: float) -> np.ndarray:
    """``prim(5, N)`` filled with the freestream (initial_conditions.f90:18-22)."""
    return np.tile(np.array(freestream(mach, aoa_deg), dtype=np.float64), (n, 1))


# The generators use only operations whose results do not depend on the host
# CPU: IEEE +, -, *, / and sqrt (numpy rounds these exactly on every SIMD
# path), and the C library's scalar sin/cos through `math`.  numpy's
# vectorised sin/cos and BLAS products may round differently on different
# CPUs, and a cloud must be the same bits on every machine that regenerates
# it for a parity check.


def _fibonacci_sphere(m: int) -> np.ndarray:
    i = np.arange(m, dtype=np.float64) + 0.5
    zz = 1.0 - 2.0 * i / m
    rr = np.sqrt(np.maximum(0.0, 1.0 - zz * zz))
    phi = i * (math.pi * (3.0 - math.sqrt(5.0)))
    cphi = np.array([math.cos(v) for v in phi.tolist()], dtype=np.float64)
    sphi = np.array([math.sin(v) for v in phi.tolist()], dtype=np.float64)
    return np.stack([rr * cphi, rr * sphi, zz], axis=1)


def _rows_norm(v: np.ndarray) -> np.ndarray:
    """Euclidean norm of each row of an (n, 3) array, summed in a fixed order."""
    return np.sqrt(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2])


def _rotate(u: np.ndarray, rot: np.ndarray) -> np.ndarray:
    """u @ rot.T written out, so every product and sum rounds the same way."""
    out = np.empty_like(u)
    for r in range(3):
        out[:, r] = u[:, 0] * rot[r, 0] + u[:, 1] * rot[r, 1] + u[:, 2] * rot[r, 2]
    return out


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = [float(v) for v in rng.standard_normal(4)]
    nq = math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    a, b, c, d = (v / nq for v in q)
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def _boundary_frames(nor: np.ndarray):
    """Right-handed frame with the given unit normal: tan1 = z x nor (x fallback)."""
    nx, ny = nor[:, 0], nor[:, 1]
    h = np.sqrt(nx * nx + ny * ny)
    tan1 = np.zeros_like(nor)
    ok = h > 1e-12
    tan1[ok, 0] = -ny[ok] / h[ok]
    tan1[ok, 1] = nx[ok] / h[ok]
    tan1[~ok, 0] = 1.0
    tan2 = np.empty_like(nor)
    tan2[:, 0] = nor[:, 1] * tan1[:, 2] - nor[:, 2] * tan1[:, 1]
    tan2[:, 1] = nor[:, 2] * tan1[:, 0] - nor[:, 0] * tan1[:, 2]
    tan2[:, 2] = nor[:, 0] * tan1[:, 1] - nor[:, 1] * tan1[:, 0]
    tan2 /= _rows_norm(tan2)[:, None]
    return tan1, tan2


def _knn_connectivity(pts: np.ndarray, k: int, device: int = -1):
    """(nbhs, conn, min_dist): the k nearest neighbours of every point, by
    squared distance then index (the library's mfcfd_knn on the host's
    threads, or on GPU `device`: the same arrays).  min_dist is the distance
    to the nearest neighbour, evaluated
    like the solver evaluates distances (sqrt of the summed squared
    deltas)."""
    from ._lib import MfcfdError
    try:
        return knn(pts[:, 0], pts[:, 1], pts[:, 2], k, device=device)
    except MfcfdError as e:
        if "coincide" in str(e):
            raise ValueError("duplicate points in generated cloud") from e
        raise


def knn(x: np.ndarray, y: np.ndarray, z: np.ndarray, k: int = 26, device: int = -1):
    """(nbhs, conn, min_dist) of the k nearest neighbours of every point
    through the library (mfcfd_knn): on GPU `device`, or on the host's
    threads for device < 0; both give the same arrays, ordered by squared
    distance then index, as _knn_connectivity's."""
    from . import _lib
    from ._lib import MfcfdError, ptr
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    n = x.shape[0]
    nbhs = np.zeros(n, dtype=np.int32)
    conn = np.zeros((n, MAX_CONN), dtype=np.int32)
    md = np.zeros(n)
    L = _lib.lib()
    rc = L.mfcfd_knn(int(device), n, ptr(x), ptr(y), ptr(z), int(k), ptr(nbhs), ptr(conn), ptr(md))
    if rc != 0:
        raise MfcfdError(rc, L.mfcfd_last_error(None).decode())
    return nbhs, conn, md


def shell_cloud(n_shells: int, pts_per_shell: int, r0: float = 0.5,
                r1: float = 10.0, jitter: float = 0.02, k: int = 26,
                seed: int = 1001, aspect=(1.0, 1.0, 1.0),
                name: str = "sphere", knn_device: int = -1) -> PointCloud:
    """Concentric shells around a sphere or ellipsoid body.

    Shell ``s`` has radius ``r0 * (r1/r0)**(s/(n_shells-1))`` and carries a
    Fibonacci lattice of ``pts_per_shell`` points under a seeded random
    rotation.  Interior shells get a multiplicative radial jitter
    ``1 + jitter*U[-1,1]``; the wall (shell 0) and the outer boundary (last
    shell) stay on their exact surfaces.  ``aspect`` stretches the body and
    the shells into an ellipsoid with semi-axes ``aspect * r``.

    Frames: interior points use the global axes; wall and outer points use
    the outward unit normal as ``nor``, ``tan1 = z x nor`` normalised
    (x when ``nor`` is along z) and ``tan2 = nor x tan1``.  The neighbours
    are found on GPU ``knn_device`` (>= 0) or the host's threads; the cloud is
    the same either way.
    """
    if n_shells < 3:
        raise ValueError("need at least 3 shells")
    rng = np.random.Generator(np.random.PCG64(seed))
    ax = np.asarray(aspect, dtype=np.float64)
    unit = _fibonacci_sphere(pts_per_shell)
    pts, status, nors = [], [], []
    for s in range(n_shells):
        r = r0 * (r1 / r0) ** (s / (n_shells - 1))
        rot = _random_rotation(rng)
        u = _rotate(unit, rot)
        if 0 < s < n_shells - 1:
            scale = r * (1.0 + jitter * rng.uniform(-1.0, 1.0, size=pts_per_shell))
        else:
            scale = np.full(pts_per_shell, r)
        p = u * scale[:, None] * ax[None, :]
        pts.append(p)
        st = STATUS_INTERIOR
        if s == 0:
            st = STATUS_WALL
        elif s == n_shells - 1:
            st = STATUS_OUTER
        status.append(np.full(pts_per_shell, st, dtype=np.int32))
        # outward normal of the ellipsoid x^2/a^2 + ... = r^2 at p
        g = p / (ax[None, :] ** 2)
        nors.append(g / _rows_norm(g)[:, None])
    pts = np.concatenate(pts)
    status = np.concatenate(status)
    nor_b = np.concatenate(nors)
    n = pts.shape[0]
    tan1 = np.zeros((n, 3))
    tan2 = np.zeros((n, 3))
    nor = np.zeros((n, 3))
    tan1[:, 0] = 1.0
    tan2[:, 1] = 1.0
    nor[:, 2] = 1.0
    b = status != STATUS_INTERIOR
    t1b, t2b = _boundary_frames(nor_b[b])
    tan1[b], tan2[b], nor[b] = t1b, t2b, nor_b[b]
    nbhs, conn, md = _knn_connectivity(pts, k, knn_device)
    a, bb, c = ax * r0
    # Surface area of the body (Thomsen's approximation for an ellipsoid).
    pp = 1.6075
    area = 4 * math.pi * (((a * bb) ** pp + (a * c) ** pp + (bb * c) ** pp) / 3) ** (1 / pp)
    return PointCloud(status=status, x=np.ascontiguousarray(pts[:, 0]),
                      y=np.ascontiguousarray(pts[:, 1]),
                      z=np.ascontiguousarray(pts[:, 2]),
                      tan1=tan1, tan2=tan2, nor=nor, nbhs=nbhs, conn=conn,
                      min_dist=md, name=name, wall_area=area,
                      ref_area=math.pi * a * bb)


def sphere_62k(seed: int = 1001) -> PointCloud:
    """Sphere cloud of 48 shells x 1300 points (62,400 points), 2% jitter."""
    return shell_cloud(48, 1300, jitter=0.02, seed=seed, name="sphere-62k")


def sphere_1m(seed: int = 2001) -> PointCloud:
    """Sphere cloud of 96 shells x 11,500 points (1,104,000 points), 1% jitter."""
    return shell_cloud(96, 11500, jitter=0.01, seed=seed, name="sphere-1.1M")


def small_sphere(n_shells: int = 8, pts_per_shell: int = 150, seed: int = 7,
                 jitter: float = 0.02, r1: float = 1.7) -> PointCloud:
    """A small cloud of the same construction for quick parity cases.

    The outer radius is chosen so that the radial shell spacing stays below
    the in-shell point spacing, as in the 62k cloud; otherwise the 26 nearest
    neighbours of a point all lie in its own shell and some of its split
    stencils come out empty.
    """
    return shell_cloud(n_shells, pts_per_shell, r1=r1, jitter=jitter, seed=seed,
                       name=f"sphere-{n_shells}x{pts_per_shell}")


def with_supersonic_boundary(cloud: PointCloud, fraction: float = 0.3) -> PointCloud:
    """A copy of `cloud` whose outer points far upstream become supersonic
    inlet points (status 5) and those far downstream supersonic outlet points
    (status 6): x below -fraction, or above +fraction, times the outer
    radius."""
    st = cloud.status.copy()
    outer = st == STATUS_OUTER
    r = np.sqrt(cloud.x ** 2 + cloud.y ** 2 + cloud.z ** 2)
    rmax = float(r[outer].max()) if outer.any() else 1.0
    st[outer & (cloud.x < -fraction * rmax)] = STATUS_SUPERSONIC_INLET
    st[outer & (cloud.x > fraction * rmax)] = STATUS_SUPERSONIC_OUTLET
    return dataclasses.replace(cloud, status=st, name=cloud.name + "-supersonic")


def initial_state(cloud: PointCloud, mach: float, aoa_deg: float) -> np.ndarray:
    """Impulsive-start initial state ``prim(5, N)``.

    The reference starts from a stored solution (initial_conditions.f90:26);
    a uniform freestream is a fixed point of the discrete scheme (every flux
    difference vanishes), so the iteration would not move.  This start is the
    freestream everywhere except that wall points have the normal velocity
    component removed (no penetration), which is what the reference's
    explicit update imposes at the wall (state_update.f90:37).
    """
    prim = freestream_prim(cloud.n, mach, aoa_deg)
    w = cloud.status == STATUS_WALL
    u = prim[w, 1:4]
    nrm = cloud.nor[w]
    un = np.sum(u * nrm, axis=1)
    prim[w, 1:4] = u - un[:, None] * nrm
    return prim
