"""Generate the 62,400-point sphere fixture from the translated reference.

The workload is the seeded 62,400-point sphere (48 shells x 1,300 points, 2%
jitter) at Mach 0.4, alpha 0, run for 500 iterations from the impulsive
start.  The reference's own routines, translated to C by oracle/f2c_ref.py
(oracle/_ref/libref*.so), run it twice: with glibc's exp/log/erf (what the
Fortran program calls) and with the solver's own exp/log/erf (mfmath).  The
fixture keeps, for each build:

    res            (500, 2) res_new and residue of every iteration
                   (fpi_solver.f90:38-43, state_update_implicit.f90:187)
    snap_iters     iterations with a snapshot: 1, 10, 100, 500
    prim_sha256    SHA-256 of prim(5, N) (C-order (N, 5) float64 bytes)
    prim_fsum      exactly rounded sum of each prim component (math.fsum)
    cl, cd         lift and drag from the project's force definition (the
                   reference computes no forces): F = -sum over wall points
                   of (p - p_inf) A nor, A = wall area / wall points,
                   CL = F.(-sin a, cos a, 0)/q, CD = F.(cos a, sin a, 0)/q,
                   q = rho_inf |u_inf|^2 S / 2, summed with math.fsum

plus the SHA-256 of the generated cloud, so a check can tell a changed
cloud from a changed solver.  The arrays are a few KB; the cloud itself is
regenerated from its seed (mfcfd.cloud.sphere_62k).

Usage: MFCFD_REFERENCE_DIR=<reference checkout> python tests/golden/make_sphere62k.py
(about 12 minutes per build on one core; the two builds run in parallel)
"""
import hashlib
import json
import math
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "3d-mfcfd_b200"))
sys.path.insert(0, REPO)

MACH, AOA = 0.4, 0.0
ITERS = 500
SNAPS = (1, 10, 100, 500)
OUT = os.path.join(HERE, "sphere_62k_500.npz")


def cloud_sha256(c) -> str:
    h = hashlib.sha256()
    for a in (c.status, c.x, c.y, c.z, c.tan1, c.tan2, c.nor, c.nbhs, c.conn, c.min_dist):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def prim_sha256(prim: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(prim, dtype=np.float64).tobytes()).hexdigest()


def forces(c, prim, mach, aoa_deg):
    """CL, CD of prim with the project's definition, exactly summed."""
    from mfcfd import cloud as cl
    rho, u1, u2, u3, pinf = cl.freestream(mach, aoa_deg)
    wall = np.nonzero(c.status == cl.STATUS_WALL)[0]
    a_each = c.wall_area / len(wall)
    f = [math.fsum(float(-(prim[i, 4] - pinf) * a_each * c.nor[i, r]) for i in wall) for r in range(3)]
    v2 = u1 * u1 + u2 * u2
    ang = math.atan2(u2, u1)
    q = 0.5 * rho * v2 * c.ref_area
    clv = (-f[0] * math.sin(ang) + f[1] * math.cos(ang)) / q
    cdv = (f[0] * math.cos(ang) + f[1] * math.sin(ang)) / q
    return clv, cdv


def run_build(libm: str, path: str):
    """One translated-reference run (own process: the program is global)."""
    from mfcfd import cloud as cl
    from oracle import ref_translated as R
    c = cl.sphere_62k()
    prim0 = cl.initial_state(c, MACH, AOA)
    r = R.TranslatedReference(c, prim0, MACH, AOA, libm=libm)
    res, sha, fs, cls, cds = [], [], [], [], []
    for t in range(1, ITERS + 1):
        res.append(r.step(t))
        if t in SNAPS:
            p = r.get("prim")
            sha.append(prim_sha256(p))
            fs.append([math.fsum(p[:, k].tolist()) for k in range(5)])
            a, b = forces(c, p, MACH, AOA)
            cls.append(a)
            cds.append(b)
    np.savez(path, res=np.array(res), prim_sha256=np.array(sha), prim_fsum=np.array(fs),
             cl=np.array(cls), cd=np.array(cds))


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "--build":
        run_build(sys.argv[2], sys.argv[3])
        return
    from oracle import ref_translated as R
    if not R.build():
        sys.exit("set MFCFD_REFERENCE_DIR to the reference checkout to build the translated reference")
    from mfcfd import cloud as cl
    c = cl.sphere_62k()
    tmp = {b: os.path.join(HERE, f"_tmp_{b}.npz") for b in ("glibc", "mfmath")}
    procs = [subprocess.Popen([sys.executable, __file__, "--build", b, tmp[b]]) for b in tmp]
    for p in procs:
        if p.wait() != 0:
            sys.exit("a translated-reference run failed")
    data = {}
    for b, path in tmp.items():
        with np.load(path) as z:
            for k in z.files:
                data[f"{b}_{k}"] = z[k]
        os.remove(path)
    meta = {"mach": MACH, "aoa": AOA, "iters": ITERS, "snaps": list(SNAPS),
            "cloud": "sphere_62k(seed=1001)", "cloud_sha256": cloud_sha256(c), "n": c.n}
    data["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(OUT, **data)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
