"""Generate the golden fixtures from the translated reference.

The reference (Fortran) has no tests, data or fixtures, and no Fortran compiler
exists here.  oracle/f2c_ref.py translates the reference's own source files to
C; this script runs that program (oracle/_ref/libref*.so, built by
`oracle.ref_translated.build()` from the reference checkout) on small seeded
clouds and stores its outputs:

    sphere_600.npz  cloud arrays, initial state, and for each case
                    (Mach, alpha) = (0.4, 0), (0.8, 2):
                      alias / point_with_alias, split-list counts and entries,
                      every field after iteration 1, res_new/residue for 20
                      iterations and prim after 20 iterations, from the build
                      with glibc's exp/log/erf ("glibc") and the build with the
                      solver's own exp/log/erf ("mfmath").

Usage: MFCFD_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "3d-mfcfd_b200"))
sys.path.insert(0, REPO)

CASES = [(0.4, 0.0), (0.8, 2.0)]
ITERS = 20
FIELDS = ["prim", "u", "q", "qm", "dq", "delt", "flux_res", "delup", "delun"]


def golden_cloud():
    from mfcfd import cloud
    return cloud.shell_cloud(6, 100, r1=1.5, jitter=0.02, seed=11, name="sphere-600")


def run_case(libm, mach, aoa, out_path):
    """One translated-reference run (in its own process: the program is global)."""
    from mfcfd import cloud as cl
    from oracle import ref_translated as R
    c = golden_cloud()
    prim0 = cl.initial_state(c, mach, aoa)
    r = R.TranslatedReference(c, prim0, mach, aoa, libm=libm)
    out = {}
    a, p = r.alias()
    out["alias"], out["point_with_alias"] = a, p
    res = []
    for t in range(1, ITERS + 1):
        res.append(r.step(t))
        if t == 1:
            for f in FIELDS:
                out["it1_" + f] = r.get(f)
    out["res"] = np.array(res)
    out["prim_final"] = r.get("prim")
    np.savez(out_path, **out)


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "--case":
        libm, mach, aoa, path = sys.argv[2], float(sys.argv[3]), float(sys.argv[4]), sys.argv[5]
        run_case(libm, mach, aoa, path)
        return
    from oracle import ref_translated as R
    if not R.build():
        sys.exit("set MFCFD_REFERENCE_DIR to the reference checkout to build the translated reference")
    c = golden_cloud()
    from mfcfd import cloud as cl
    data = {"status": c.status, "x": c.x, "y": c.y, "z": c.z, "tan1": c.tan1, "tan2": c.tan2,
            "nor": c.nor, "nbhs": c.nbhs, "conn": c.conn, "min_dist": c.min_dist}
    tmp = os.path.join(HERE, "_tmp_case.npz")
    for ci, (mach, aoa) in enumerate(CASES):
        data[f"case{ci}_prim0"] = cl.initial_state(c, mach, aoa)
        for libm in ("glibc", "mfmath"):
            subprocess.run([sys.executable, __file__, "--case", libm, str(mach), str(aoa), tmp],
                           check=True)
            with np.load(tmp) as z:
                for k in z.files:
                    data[f"case{ci}_{libm}_{k}"] = z[k]
            os.remove(tmp)
    # split lists as stored by the reference, from the C++ oracle (itself
    # checked against the translated program's alias and fields)
    from oracle.oracle import Oracle
    o = Oracle(c, CASES[0][0], CASES[0][1])
    counts, lists = o.stencils(27)
    data["split_counts"], data["split_lists"] = counts, lists
    meta = {"cases": CASES, "iters": ITERS, "fields": FIELDS,
            "cloud": "shell_cloud(6, 100, r1=1.5, jitter=0.02, seed=11)"}
    data["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, "sphere_600.npz"), **data)
    print("wrote", os.path.join(HERE, "sphere_600.npz"))


if __name__ == "__main__":
    main()
