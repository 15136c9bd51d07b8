"""The multi-GPU replica protocol of bench.py on CPU: two gloo ranks, each
running its own seeded solve (the CPU oracle stands in for the GPU solver),
a barrier around the timed region and the max over ranks of the times."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import sys
    import time
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(repo, "3d-mfcfd_b200"))
    sys.path.insert(0, repo)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from mfcfd import cloud, replicas
    from oracle.oracle import Oracle
    r, w = replicas.init("gloo", timeout_s=60)
    c = cloud.shell_cloud(4, 60, r1=1.4, seed=replicas.replica_seed(100, r))
    o = Oracle(c, 0.4, 0.0)
    o.set_prim(cloud.initial_state(c, 0.4, 0.0))
    replicas.barrier()
    t0 = time.perf_counter()
    res = [o.step(t)[0] for t in (1, 2)]
    dt = time.perf_counter() - t0 + 0.05 * r          # rank 1 is the slower one
    replicas.barrier()
    dmax = replicas.max_over_ranks(dt)
    q.put((r, w, dt, dmax, c.n, res[0], float(c.x[0])))
    replicas.finalize()


def test_two_rank_replicas():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, t0, m0, n0, res0, x0), (r1, w1, t1, m1, n1, res1, x1) = out
    assert w0 == w1 == 2
    assert m0 == m1 == max(t0, t1)
    assert x0 != x1                      # distinct seeded clouds per rank
    from mfcfd.replicas import throughput
    assert throughput(n0, 2, m0, 2) == 2 * n0 * 2 / m0
