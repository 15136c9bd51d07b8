"""Iterations launched as captured CUDA graphs (mfcfd_params.graphs: 1, the
default, in batches; 2 also for single handles) against the same iterations
launched kernel by kernel: identical
bits for every schedule and precision, for chunks of odd and even length
(the U/q buffers alternate), single steps, batches, profiling (which
launches directly) and a schedule replaced by the autotuner (which drops the
captured graphs)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(c, graphs, **kw):
    from mfcfd import _lib
    from mfcfd.solver import Solver
    s = Solver(c, 0.8, 2.0, graphs=graphs, **kw)
    s.initial_conditions()
    h = [s.q_lskum(7), s.q_lskum(4, t0=8), np.array([s.fpi_solver(12), s.fpi_solver(13)])]
    s.set_profiling(True)
    h.append(s.q_lskum(2, t0=14))
    s.set_profiling(False)
    h.append(s.q_lskum(5, t0=16))
    out = (np.vstack(h), s.get(_lib.FIELD_PRIM), s.get(_lib.FIELD_DELUN))
    s.close()
    return out


@pytest.mark.parametrize("kw", [{}, {"precision": 1}, {"sweep_mode": 0}, {"sweep_mode": 1}, {"inner_iterations": 1}])
def test_graphs_equal_direct_launches(mfcfd_lib, small_cloud, kw):
    a = _run(small_cloud, 0, **kw)
    b = _run(small_cloud, 2, **kw)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_graphs_in_batches_and_after_tuning(mfcfd_lib):
    from mfcfd import _lib, batch, cloud
    from mfcfd.solver import Solver
    clouds = [cloud.small_sphere(6, 100, r1=1.5, seed=3), cloud.small_sphere(8, 150, seed=4)]
    res = {}
    for g in (0, 1):
        ss = []
        for c in clouds:
            s = Solver(c, 0.6, 1.0, graphs=g)
            s.initial_conditions()
            ss.append(s)
        h1 = batch.run_batch(ss, 6)
        ss[1].tune_chain([24, 48], iters=1)
        h2 = batch.run_batch(ss, 5)
        res[g] = (h1, h2, [s.get(_lib.FIELD_PRIM) for s in ss])
        for s in ss:
            s.close()
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
    assert all(np.array_equal(x, y) for x, y in zip(res[0][2], res[1][2]))
