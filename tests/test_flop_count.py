"""The FP64 operation counts that bench.py quotes come from the oracle built
with counting arithmetic (oracle/oracle_flops.cpp).  The counted build must
compute the same bits as the plain oracle, and its per-phase counts on the
62,400-point sphere must be the constants in bench.py."""
import numpy as np


def test_counting_build_computes_the_same_bits(oracle_lib):
    import ctypes
    from mfcfd import cloud
    c = cloud.small_sphere()
    prim0 = cloud.initial_state(c, 0.8, 2.0)
    o = oracle_lib.Oracle(c, 0.8, 2.0, libm=oracle_lib.LIBM_MFMATH)
    o.set_prim(prim0)
    for t in (1, 2, 3):
        o.step(t)
    want = o.get(oracle_lib.FIELD_PRIM)
    L = ctypes.CDLL(oracle_lib._FLOPS_LIB_PATH)
    vp = ctypes.c_void_p
    L.oracle_create.restype = vp
    L.oracle_create.argtypes = [ctypes.POINTER(oracle_lib._Params), ctypes.c_int] + [vp] * 10
    L.oracle_set_prim.argtypes = [vp, vp]
    L.oracle_fpi_step.argtypes = [vp, ctypes.c_int, vp, vp]
    L.oracle_get.argtypes = [vp, ctypes.c_int, vp]
    L.oracle_destroy.argtypes = [vp]
    h = L.oracle_create(ctypes.byref(o.params), c.n, *[oracle_lib._ptr(a) for a in o._keep])
    p0 = np.ascontiguousarray(prim0)
    L.oracle_set_prim(h, oracle_lib._ptr(p0))
    L.oracle_set_libm(1)
    r = np.zeros(2)
    for t in (1, 2, 3):
        L.oracle_fpi_step(h, t, oracle_lib._ptr(r[0:1]), oracle_lib._ptr(r[1:2]))
    got = np.empty((c.n, 5))
    L.oracle_get(h, 0, oracle_lib._ptr(got))
    L.oracle_destroy(h)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


def test_bench_flop_constants_match_the_count(oracle_lib):
    import bench
    from mfcfd import cloud
    c = cloud.sphere_62k()
    fc = oracle_lib.flop_counts(c, 0.4, 0.0, iters=1, skip=2)
    per = {k: oracle_lib.flops_of(v) / c.n for k, v in fc.items()}
    want = {"qderiv": per["qderiv_delt"], "flux": per["flux"], "dinv": per["dinv"],
            "sweep_fwd": per["sweep_fwd"], "sweep_bwd": per["sweep_bwd"],
            "update": per["update"] + per["conserved_q"], "residual": 0.0}
    got = bench.PHASE_FLOPS["sphere-62k"]
    for k, v in want.items():
        assert abs(got[k] - v) <= 0.05 + 1e-6 * v, (k, got[k], v)
    # the reference's second D_inv evaluation (backward sweep) is what is left out
    assert abs(per["other"] - per["dinv"]) <= 1e-3 * per["dinv"]
