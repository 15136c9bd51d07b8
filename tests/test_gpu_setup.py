"""Set-up passes on the GPU (mfcfd_params.gpu_setup = 1) against the host.

Split stencils, the alias search and the sweep levels must equal the host
path's exactly; the host path itself is pinned against the translated
reference (tests/test_translated_reference.py, tests/test_topology.py).
A split capacity the lists overflow makes the GPU pass hand the storage back
to the host's sequential order, which must still give the same result.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _topology(c, **params):
    from mfcfd.solver import Solver
    s = Solver(c, 0.8, 2.0, **params)
    out = {"stencils": s.stencils(27), "alias": s.alias(), "fwd": s.levels(0), "bwd": s.levels(1),
           "info": s.info()}
    s.close()
    return out


def _clouds():
    from mfcfd import cloud
    return {
        "small": cloud.small_sphere(),
        "supersonic": cloud.with_supersonic_boundary(cloud.small_sphere(7, 120, r1=1.6, seed=5)),
        "ellipsoid": cloud.shell_cloud(14, 900, r1=3.0, seed=77, aspect=(1.0, 1.8, 2.6)),
        "72k": cloud.shell_cloud(12, 6000, r1=3.0, seed=4242),
    }


@pytest.mark.parametrize("name", ["small", "supersonic", "ellipsoid", "72k"])
@pytest.mark.parametrize("extra", [{}, {"split_capacity": 20}, {"split_capacity": 12}, {"sweep_variant": 1}])
def test_gpu_setup_equals_host(mfcfd_lib, name, extra):
    from mfcfd._lib import MfcfdError
    c = _clouds()[name]
    try:
        host = _topology(c, device=-1, **extra)
    except MfcfdError as e:        # overflowing lists that name too many points
        with pytest.raises(MfcfdError) as g:
            _topology(c, device=0, gpu_setup=1, **extra)
        assert str(g.value) == str(e)
        return
    gpu = _topology(c, device=0, gpu_setup=1, **extra)
    for a, b in zip(host["stencils"], gpu["stencils"]):
        assert np.array_equal(a, b)
    for a, b in zip(host["alias"], gpu["alias"]):
        assert np.array_equal(a, b)
    assert np.array_equal(host["fwd"], gpu["fwd"]) and np.array_equal(host["bwd"], gpu["bwd"])
    for k in ("n_levels_forward", "n_levels_backward", "max_level_width", "split_overflows"):
        assert host["info"][k] == gpu["info"][k], k
    if extra.get("split_capacity") == 20:
        assert gpu["info"]["split_overflows"] > 0   # the host storage order was used


def test_gpu_setup_iterations_bitexact(mfcfd_lib):
    """A handle set up on the GPU iterates to the same bits."""
    from mfcfd import _lib, cloud
    from mfcfd.solver import Solver
    c = cloud.small_sphere(8, 150, seed=4)
    out = []
    for g in (0, 1):
        s = Solver(c, 0.8, 2.0, gpu_setup=g)
        s.initial_conditions()
        h = s.q_lskum(10)
        out.append((h, s.get(_lib.FIELD_PRIM)))
        s.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
