"""The reference program end to end: ``python -m mfcfd.program DIR``.

Mirrors meshfree_solver.f90:20-37 in a run directory: read ``3d_input_data``
(all records, or the first --max-points), read the initial state from
``stored-solution.dat``, run the q_lskum loop on the GPU writing
``residue.dat`` (q_lskum.f90:22-32), then ``print_primal_output``.  The flow
constants of parameter.f90 (Mach, angle of attack, iteration count) are
options instead of compile-time parameters.
"""
from __future__ import annotations

import argparse
import os
import sys

from . import io
from .solver import Solver


def run(directory: str, mach: float, aoa: float, max_iters: int, max_points: int | None = None,
        device: int = 0, chunk: int = 100, echo: bool = True, **params) -> Solver:
    inp = os.path.join(directory, "3d_input_data")
    cloud = io.read_input_point_data(inp, max_points)
    counts = cloud.counts()
    if echo:
        print(cloud.n)
        print(counts["wall"], counts["outer"], counts["interior"])
        print(counts["supersonic_inlet"], counts["supersonic_outlet"])
    s = Solver(cloud, mach, aoa, device=device, **params)
    s.initial_conditions(io.read_stored_solution(os.path.join(directory, "stored-solution.dat"), cloud.n))
    res_path = os.path.join(directory, "residue.dat")
    t = 1
    first = True
    while t <= max_iters:
        k = min(chunk, max_iters - t + 1)
        hist = s.q_lskum(k, t0=t)
        io.write_residue(res_path, t, hist, append=not first)
        if echo:
            for j in range(k):
                print(t + j, hist[j, 0], hist[j, 1])
        first = False
        t += k
    s.print_primal_output(directory)
    return s


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("directory")
    ap.add_argument("--mach", type=float, required=True)
    ap.add_argument("--aoa", type=float, default=0.0)
    ap.add_argument("--iters", type=int, default=1000)
    ap.add_argument("--max-points", type=int, default=None)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    s = run(a.directory, a.mach, a.aoa, a.iters, a.max_points, a.device)
    s.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
