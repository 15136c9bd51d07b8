"""The C ABI library: loads without a GPU, exports every symbol the header
declares, and reports errors as status codes."""
import ctypes
import os
import re

import numpy as np
import pytest

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "mfcfd.h")


def header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*)\s*(mfcfd_\w+)\s*\(", text, re.M)))


def test_exports_every_declared_symbol(mfcfd_lib):
    L = mfcfd_lib.lib()
    declared = header_functions()
    assert len(declared) >= 18
    for name in declared:
        assert hasattr(L, name), name
    assert set(declared) == set(mfcfd_lib.EXPORTS)


def test_params_init_matches_parameter_module(mfcfd_lib):
    from mfcfd.solver import params_for
    import math
    p = params_for(0.8, 2.0)
    theta = 2.0 * (4.0 * math.atan(1.0)) / 180.0
    assert p.power == 0.0 and p.vl_const == 2.0 and p.cfl == 5.0 and p.inner_iterations == 0
    assert p.rho_inf == 1.0 and p.pr_inf == 1.0 / 1.4 and p.u3_inf == 0.0
    assert p.u1_inf == 0.8 * math.cos(theta) and p.u2_inf == 0.8 * math.sin(theta)
    assert p.split_capacity == 22 and p.sweep_mode == 2   # MFCFD_SWEEP_CHAINS


def test_strerror(mfcfd_lib):
    L = mfcfd_lib.lib()
    assert L.mfcfd_strerror(0) == b"ok"
    assert L.mfcfd_strerror(8) == b"device wait timed out"
    assert L.mfcfd_strerror(99) == b"unknown error"


def _create(mfcfd_lib, cloud, **over):
    from mfcfd.solver import Solver
    return Solver(cloud, 0.4, 0.0, device=-1, **over)


def test_bad_inputs_are_status_codes(mfcfd_lib, small_cloud):
    import copy
    from mfcfd._lib import MfcfdError
    c = copy.deepcopy(small_cloud)
    c.status = c.status.copy()
    c.status[5] = 7
    with pytest.raises(MfcfdError) as e:
        _create(mfcfd_lib, c)
    assert e.value.code == 1 and "status" in str(e.value)
    c = copy.deepcopy(small_cloud)
    c.conn = c.conn.copy()
    c.conn[3, 0] = c.n + 5
    with pytest.raises(MfcfdError) as e:
        _create(mfcfd_lib, c)
    assert e.value.code == 1
    c = copy.deepcopy(small_cloud)
    c.status = c.status.copy()
    c.status[10] = 7
    with pytest.raises(MfcfdError) as e:
        _create(mfcfd_lib, c)
    assert e.value.code == 1
    with pytest.raises(MfcfdError) as e:
        _create(mfcfd_lib, small_cloud, power=-1.0)
    assert e.value.code == 1
    with pytest.raises(MfcfdError) as e:
        _create(mfcfd_lib, small_cloud, precision=3)
    assert e.value.code == 6
    for prec in (1, 2):                           # mixed precision: chain schedule only
        with pytest.raises(MfcfdError) as e:
            _create(mfcfd_lib, small_cloud, precision=prec, sweep_mode=0)
        assert e.value.code == 6
    with pytest.raises(MfcfdError) as e:
        _create(mfcfd_lib, small_cloud, storage_order=2)
    assert e.value.code == 1
    with pytest.raises(MfcfdError) as e:
        _create(mfcfd_lib, small_cloud, sweep_mode=3)
    assert e.value.code == 1
    with pytest.raises(MfcfdError) as e:
        _create(mfcfd_lib, small_cloud, inner_iterations=-1)
    assert e.value.code == 1


def test_host_only_handle_refuses_device_calls(mfcfd_lib, small_cloud):
    from mfcfd._lib import MfcfdError
    s = _create(mfcfd_lib, small_cloud)
    with pytest.raises(MfcfdError):
        s.initial_conditions()
    with pytest.raises(MfcfdError):
        s.residual_noalloc()
    assert s.info()["n_points"] == small_cloud.n
    # a group needs handles with device state, at most MFCFD_GROUP_MAX_CLOUDS
    import ctypes
    import numpy as np
    from mfcfd import _lib
    t0 = np.ones(40, dtype=np.int32)
    for count in (0, 1, _lib.GROUP_MAX_CLOUDS + 1):
        hs = (ctypes.c_void_p * 40)(*([s.h.value] * 40))
        assert _lib.lib().mfcfd_run_group(hs, count, _lib.ptr(t0), 1, None, None) == 1
    assert _lib.lib().mfcfd_run_group(None, 1, _lib.ptr(t0), 1, None, None) == 1


def test_prepare_needs_a_device_and_serving_helpers(mfcfd_lib, small_cloud):
    """mfcfd_prepare refuses a host-only handle; the serving statistics; a
    server configuration without set-up threads is refused."""
    from mfcfd import _lib, serve
    from mfcfd.solver import params_for
    L = _lib.lib()
    p = params_for(0.8, 2.0, device=-1)
    h = ctypes.c_void_p()
    z = ctypes.c_void_p(0)
    assert L.mfcfd_prepare(ctypes.byref(p), small_cloud.n, *([z] * 10), ctypes.byref(h)) == 1
    assert not h.value
    t = serve.poisson_arrivals(20.0, 2000, seed=5)
    assert np.all(np.diff(t) > 0) and abs(2000 / t[-1] - 20.0) < 2.0
    s = serve.latency_summary([1.0, 2.0, 3.0, 4.0])
    assert s["p50"] == 2.5 and abs(s["p99"] - 3.97) < 1e-9 and s["max"] == 4.0
    cfg = _lib.ServerConfig(device=0, max_live=0, setup_threads=0, chunk=10)
    srv = ctypes.c_void_p()
    assert L.mfcfd_server_create(ctypes.byref(cfg), ctypes.byref(srv)) == 1
    cfg = _lib.ServerConfig(device=0, max_live=0, setup_threads=2, chunk=10, device_setup=2)
    assert L.mfcfd_server_create(ctypes.byref(cfg), ctypes.byref(srv)) == 1
    # the connectivity search checks its arguments before touching a device
    x = np.zeros(4)
    nb, cn, md = np.zeros(4, np.int32), np.zeros((4, 27), np.int32), np.zeros(4)
    assert L.mfcfd_knn(0, 4, _lib.ptr(x), _lib.ptr(x), _lib.ptr(x), 28, _lib.ptr(nb), _lib.ptr(cn),
                       _lib.ptr(md)) == 1
    assert L.mfcfd_knn(0, 4, _lib.ptr(x), _lib.ptr(x), _lib.ptr(x), 3, None, _lib.ptr(cn), _lib.ptr(md)) == 1


def test_host_memory_exhaustion_is_a_status_not_a_crash():
    """No exception crosses the C ABI: with the process's address space
    capped just above what it uses, a 72k-point set-up (worker threads and
    large tables) returns MFCFD_ERR_NOMEM with a message, and the process
    goes on."""
    import subprocess
    import sys
    import textwrap
    script = textwrap.dedent('''
        import ctypes, resource, sys
        sys.path.insert(0, sys.argv[1])
        from mfcfd import _lib, cloud
        from mfcfd._lib import ptr
        from mfcfd.serve import _cloud_arrays
        from mfcfd.solver import params_for
        c = cloud.shell_cloud(12, 6000, r1=3.0, seed=4242)
        arrs = _cloud_arrays(c)
        L = _lib.lib()
        p = params_for(0.4, 0.0, device=-1)
        h = ctypes.c_void_p()
        vm = int(open("/proc/self/statm").read().split()[0]) * resource.getpagesize()
        soft, hard = resource.getrlimit(resource.RLIMIT_AS)
        resource.setrlimit(resource.RLIMIT_AS, (vm + (32 << 20), hard))
        rc = L.mfcfd_create(ctypes.byref(p), c.n, *[ptr(a) for a in arrs], ctypes.byref(h))
        resource.setrlimit(resource.RLIMIT_AS, (soft, hard))
        msg = L.mfcfd_last_error(h).decode() if h.value else ""
        if h.value:
            L.mfcfd_destroy(h)
        print(rc, msg)
    ''')
    import os
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "3d-mfcfd_b200")
    out = subprocess.run([sys.executable, "-c", script, pkg], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    rc, _, msg = out.stdout.strip().partition(" ")
    assert int(rc) == 7, out.stdout
    assert "host" in msg, msg
