"""Invariants of the chain schedule the sweep kernel relies on, checked on
the host (tests/chain_schedule_check.cpp, built with csrc/mfcfd_setup.cpp):
every swept point once per direction in level order, same-warp producers
first, ring terms within the warp's last points at the right slot, every
other producer a shared consumer reads marked to publish, the g0 marks of
the points whose phase A runs before the sweeps, and a deterministic
(parallel) build.  Needs g++ and the CUDA headers, no GPU."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "3d-mfcfd_b200", "csrc")
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")

pytestmark = pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC),
                                reason="needs g++ and the CUDA headers")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("chain") / "chain_schedule_check")
    subprocess.run(["g++", "-O1", "-std=c++17", "-pthread", "-ffp-contract=off", "-I", CSRC, "-I", CUDA_INC,
                    os.path.join(ROOT, "tests", "chain_schedule_check.cpp"), os.path.join(CSRC, "mfcfd_setup.cpp"),
                    "-o", exe], check=True, capture_output=True, text=True)
    return exe


def _check(checker, tmp_path, c, warps, variant=0, env=None):
    for name, a, t in (("status", c.status, np.int32), ("x", c.x, np.float64), ("y", c.y, np.float64),
                       ("z", c.z, np.float64), ("tan1", c.tan1, np.float64), ("tan2", c.tan2, np.float64),
                       ("nor", c.nor, np.float64), ("nbhs", c.nbhs, np.int32), ("conn", c.conn, np.int32),
                       ("md", c.min_dist, np.float64)):
        np.ascontiguousarray(a, dtype=t).tofile(str(tmp_path / f"{name}.bin"))
    out = subprocess.run([checker, str(tmp_path), str(c.n), str(warps), str(variant)], capture_output=True,
                         text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stdout + out.stderr
    return out.stdout


@pytest.mark.parametrize("warps", [-200, -100, -75, 7])
def test_schedule_invariants_small_sphere(checker, tmp_path, small_cloud, warps):
    out = _check(checker, tmp_path, small_cloud, warps)
    assert out.startswith("ok") and " g0 0" not in out


@pytest.mark.parametrize("variant", [0, 1])
def test_schedule_invariants_supersonic_and_backup_driver(checker, tmp_path, variant):
    from mfcfd import cloud
    c = cloud.with_supersonic_boundary(cloud.small_sphere(7, 120, r1=1.6, seed=5))
    assert _check(checker, tmp_path, c, -200, variant).startswith("ok")


def test_schedule_invariants_threaded_build(checker, tmp_path):
    """15,000 points: the set-up passes and the term marking run on several
    host threads, and every table and the schedule are the same bytes as with
    one thread (MFCFD_SETUP_THREADS=1)."""
    from mfcfd import cloud
    c = cloud.shell_cloud(10, 1500, r1=2.0, seed=77)
    outs = []
    for threads in ("1", "4", "16"):
        env = dict(os.environ, MFCFD_SETUP_THREADS=threads)
        out = _check(checker, tmp_path, c, -100, env=env)
        assert out.startswith("ok")
        outs.append(out.split("hash")[1].strip())
    assert outs[0] == outs[1] == outs[2]
