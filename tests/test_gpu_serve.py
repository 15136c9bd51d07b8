"""Request server (mfcfd_server_*): continuous batching of steady-state solves.

Each served result must be the same as the request solved alone, bit for bit:
the server runs every request in whole rounds of `chunk` iterations from
t = 1, and a batch of handles computes exactly what each handle computes on
its own.  Admission must keep the live requests' device memory within the
budget, and requests that arrive while others iterate are admitted as memory
frees up.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases():
    from mfcfd import _lib, cloud
    return [
        (cloud.small_sphere(8, 150, seed=4), 0.8, 2.0, {}),
        (cloud.small_sphere(6, 100, r1=1.5, seed=3), 0.4, 0.0, {}),
        (cloud.small_sphere(10, 160, r1=1.9, seed=9), 0.6, -3.0, {"precision": _lib.PRECISION_MIXED}),
        (cloud.with_supersonic_boundary(cloud.small_sphere(7, 120, r1=1.6, seed=5)), 0.7, 1.0, {}),
    ]


@pytest.mark.parametrize("target,max_iters", [(-1.0, 200), (-6.0, 30)])
def test_results_equal_alone_and_in_the_mix(mfcfd_lib, target, max_iters):
    from mfcfd import serve
    chunk = 10
    cases = _cases()
    with serve.Server(chunk=chunk, setup_threads=2) as srv:
        ids = [srv.submit(c, m, a, max_iters=max_iters, residue_target=target, **kw) for c, m, a, kw in cases]
        res = [srv.wait(i, timeout=300) for i in ids]
        st = srv.stats()
    assert st["completed"] == len(cases) and st["failed"] == 0 and st["live"] == 0
    assert st["peak_live"] >= 2            # they did share the device
    # utilisation: busy time and held slots accumulate; a request runs only
    # between its admission and its retirement
    assert st["slot_capacity"] > 0 and 0 < st["busy_s"] and 0 < st["slot_s"]
    assert st["slot_s"] <= st["slot_capacity"] * st["busy_s"] * (1 + 1e-9)
    for (c, m, a, kw), r in zip(cases, res):
        alone = serve.solve_alone(c, m, a, chunk, max_iters, target, **kw)
        assert r["status"] == 0
        assert 0 < r["run_s"] <= r["t_done"] - r["t_admit"]
        assert r["iters"] == alone["iters"] and bool(r["converged"]) == alone["converged"]
        assert np.array_equal(r["prim"], alone["prim"])
        assert r["res_new"] == alone["res_new"] and r["residue"] == alone["residue"]
        assert r["cl"] == alone["cl"] and r["cd"] == alone["cd"]
        if target > -2:
            assert r["converged"] and r["iters"] < max_iters and r["residue"] <= target
        else:
            assert not r["converged"] and r["iters"] == max_iters


def test_admission_by_device_memory(mfcfd_lib):
    """A budget that fits one request at a time serialises them; a request
    larger than the budget fails with MFCFD_ERR_NOMEM and harms no other."""
    from mfcfd import cloud, serve
    c = cloud.small_sphere(8, 150, seed=4)
    b = serve.device_bytes(c, 0.8, 2.0)
    big = cloud.small_sphere(12, 400, r1=2.2, seed=6)
    assert serve.device_bytes(big, 0.8, 2.0) > int(1.5 * b)
    # chain_percent 0: each request keeps the schedule device_bytes measured
    with serve.Server(chunk=10, hbm_budget=int(1.5 * b), chain_percent=0) as srv:
        ids = [srv.submit(c, 0.8, 2.0, max_iters=20, residue_target=-9.0) for _ in range(3)]
        bad = srv.submit(big, 0.8, 2.0, max_iters=20)
        res = [srv.wait(i, timeout=300) for i in ids]
        rb = srv.wait(bad, timeout=300)
        st = srv.stats()
    assert rb["status"] == 7
    assert all(r["status"] == 0 and r["iters"] == 20 and r["device_bytes"] == b for r in res)
    assert st["peak_live"] == 1 and st["peak_bytes_live"] <= int(1.5 * b)
    assert all(np.array_equal(r["prim"], res[0]["prim"]) for r in res)
    order = sorted(res, key=lambda r: r["t_admit"])
    for a, bb in zip(order, order[1:]):
        assert bb["t_admit"] >= a["t_done"] - 1e-3   # admitted once the previous one retired


def test_requests_arriving_while_others_iterate(mfcfd_lib):
    from mfcfd import cloud, serve
    c1, c2 = cloud.small_sphere(8, 150, seed=4), cloud.small_sphere(6, 100, r1=1.5, seed=3)
    with serve.Server(chunk=5, setup_threads=1) as srv:
        first = srv.submit(c1, 0.8, 2.0, max_iters=300, residue_target=-9.0)
        deadline = time.time() + 60
        while srv.stats()["live"] < 1 and time.time() < deadline:
            time.sleep(0.01)
        assert srv.stats()["live"] == 1
        late = [srv.submit(c2, 0.4, 0.0, max_iters=20, residue_target=-9.0) for _ in range(2)]
        rl = [srv.wait(i, timeout=300) for i in late]
        rf = srv.wait(first, timeout=300)
        st = srv.stats()
    assert rf["status"] == 0 and rf["iters"] == 300
    # the late requests joined the running one and finished before it
    assert all(r["t_admit"] < rf["t_done"] and r["t_done"] < rf["t_done"] for r in rl)
    assert st["peak_live"] >= 2
    assert np.array_equal(rl[0]["prim"], rl[1]["prim"])


def test_default_initial_state_is_the_impulsive_start(mfcfd_lib):
    """A request submitted without a state through the C ABI starts from the
    freestream with the wall-normal velocity removed, as cloud.initial_state."""
    import ctypes
    from mfcfd import _lib, cloud, serve
    from mfcfd.solver import params_for
    c = cloud.small_sphere(6, 100, r1=1.5, seed=3)
    arrs = serve._cloud_arrays(c)
    q = _lib.Request()
    q.params = params_for(0.8, 2.0)
    q.n = c.n
    for name, a in zip(("status", "x", "y", "z", "tan1", "tan2", "nor", "nbhs", "conn", "min_dist"), arrs):
        setattr(q, name, a.ctypes.data)
    q.prim = None
    q.max_iters = 10
    q.residue_target = -9.0
    with serve.Server(chunk=10) as srv:
        rid = ctypes.c_int64()
        assert _lib.lib().mfcfd_server_submit(srv.h, ctypes.byref(q), ctypes.byref(rid)) == 0
        srv._n[rid.value] = c.n
        r = srv.wait(rid.value, timeout=100)
        r2 = srv.wait(srv.submit(c, 0.8, 2.0, max_iters=10, residue_target=-9.0, forces=False), timeout=100)
    assert r["status"] == 0 and np.allclose(r["prim"], r2["prim"], rtol=1e-12, atol=1e-14)


def test_malformed_request_fails_alone(mfcfd_lib):
    """A request whose connectivity names a point that does not exist
    fails in set-up with MFCFD_ERR_ARG; the requests beside it complete
    with the same bits as alone."""
    import copy
    from mfcfd import cloud, serve
    good = cloud.small_sphere(6, 100, r1=1.5, seed=3)
    bad = copy.deepcopy(good)
    bad.conn = bad.conn.copy()
    bad.conn[5, 0] = bad.n + 7
    with serve.Server(chunk=10) as srv:
        ids = [srv.submit(good, 0.6, 1.0, max_iters=20, residue_target=-9.0),
               srv.submit(bad, 0.6, 1.0, max_iters=20, residue_target=-9.0),
               srv.submit(good, 0.6, 1.0, max_iters=20, residue_target=-9.0)]
        res = [srv.wait(i, timeout=120) for i in ids]
        st = srv.stats()
    assert res[1]["status"] == 1 and "prim" not in res[1]
    assert res[0]["status"] == 0 and res[2]["status"] == 0
    assert np.array_equal(res[0]["prim"], res[2]["prim"])
    assert st["failed"] == 1 and st["completed"] == 2
    alone = serve.solve_alone(good, 0.6, 1.0, 10, 20, -9.0)
    assert np.array_equal(res[0]["prim"], alone["prim"])


def test_device_setup_server_equals_host_setup(mfcfd_lib):
    """device_setup = 1: requests set up on the device at admission give the
    same results as the host-prepared server's (the set-up arrays are the
    same bytes); the supersonic request falls back to the host set-up inside
    mfcfd_create.  The reservation becomes the handle's own bytes, and every
    byte is released at the end."""
    from mfcfd import serve
    chunk = 10
    cases = _cases()
    out = []
    for dev in (False, True):
        with serve.Server(chunk=chunk, setup_threads=2, device_setup=dev) as srv:
            ids = [srv.submit(c, m, a, max_iters=60, residue_target=-1.0, **kw) for c, m, a, kw in cases]
            res = [srv.wait(i, timeout=300) for i in ids]
            st = srv.stats()
        assert st["completed"] == len(cases) and st["failed"] == 0 and st["live"] == 0
        assert st["bytes_live"] == 0
        out.append(res)
    for a, b in zip(*out):
        assert a["status"] == b["status"] == 0
        assert a["iters"] == b["iters"]
        assert np.array_equal(a["prim"], b["prim"])
        assert a["cl"] == b["cl"] and a["cd"] == b["cd"]
    for (c, _, _, _), b in zip(cases, out[1]):
        assert b["device_bytes"] > 0
