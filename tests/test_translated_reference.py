"""Rebuild the translated reference from the reference sources (where the
checkout exists) and check it still produces the committed fixtures."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

REF = os.environ.get("MFCFD_REFERENCE_DIR", "")
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "sphere_600.npz")

@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="MFCFD_REFERENCE_DIR is not set")
def test_translation_reproduces_fixtures(tmp_path):
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, repo)
    from oracle import ref_translated as R
    assert R.build(REF)
    out = tmp_path / "case.npz"
    with np.load(GOLDEN) as z:
        g = {k: z[k] for k in z.files}
    meta = json.loads(str(g["meta"]))
    mach, aoa = meta["cases"][1]
    subprocess.run([sys.executable, os.path.join(repo, "tests", "golden", "make_golden.py"),
                    "--case", "glibc", str(mach), str(aoa), str(out)], check=True)
    with np.load(out) as z:
        assert np.array_equal(z["res"], g["case1_glibc_res"])
        assert np.array_equal(z["prim_final"], g["case1_glibc_prim_final"])


def test_oracle_inner_iterations_match_translated_reference(oracle_lib):
    """inner_iterations > 0 (q_derivatives.f90:116-201): the restatement and
    the reference's own routines agree bit for bit (glibc libm both sides)."""
    import numpy as np
    from mfcfd import cloud
    from oracle import ref_translated
    if not ref_translated.available("glibc"):
        import pytest
        pytest.skip("translated reference not built")
    c = cloud.small_sphere(6, 100, r1=1.5)
    p0 = cloud.initial_state(c, 0.8, 2.0)
    r = ref_translated.TranslatedReference(c, p0, 0.8, 2.0, inner_iterations=2)
    o = oracle_lib.Oracle(c, 0.8, 2.0, inner_iterations=2)
    o.set_prim(p0)
    for t in range(1, 4):
        assert r.step(t) == o.step(t)
    assert np.array_equal(r.get("dq"), o.get(oracle_lib.FIELD_DQ))
    assert np.array_equal(r.get("prim"), o.get(oracle_lib.FIELD_PRIM))
    ref_translated.TranslatedReference(c, p0, 0.8, 2.0)   # back to the default


def test_oracle_supersonic_points_match_translated_reference(oracle_lib):
    """Status 5/6 points: the restatement and the reference's own routines
    agree bit for bit (glibc libm both sides)."""
    import numpy as np
    import pytest
    from mfcfd import cloud
    from oracle import ref_translated
    if not ref_translated.available("glibc"):
        pytest.skip("translated reference not built")
    c = cloud.with_supersonic_boundary(cloud.small_sphere(6, 100, r1=1.5))
    p0 = cloud.initial_state(c, 0.8, 2.0)
    r = ref_translated.TranslatedReference(c, p0, 0.8, 2.0)
    o = oracle_lib.Oracle(c, 0.8, 2.0)
    o.set_prim(p0)
    for t in range(1, 6):
        assert r.step(t) == o.step(t)
    for name, fid in (("prim", oracle_lib.FIELD_PRIM), ("delun", oracle_lib.FIELD_DELUN),
                      ("dq", oracle_lib.FIELD_DQ), ("flux_res", oracle_lib.FIELD_FLUX_RES)):
        assert np.array_equal(r.get(name), o.get(fid)), name


@pytest.mark.parametrize("power", [2.0, 0.5])
def test_oracle_weighted_least_squares_match_translated_reference(oracle_lib, power):
    """power != 0 (parameter.f90:21): restatement and reference agree bit for bit."""
    import numpy as np
    from mfcfd import cloud
    from oracle import ref_translated
    if not ref_translated.available("glibc"):
        pytest.skip("translated reference not built")
    c = cloud.small_sphere(6, 100, r1=1.5)
    p0 = cloud.initial_state(c, 0.8, 2.0)
    r = ref_translated.TranslatedReference(c, p0, 0.8, 2.0, power=power)
    o = oracle_lib.Oracle(c, 0.8, 2.0, power=power)
    o.set_prim(p0)
    for t in range(1, 4):
        assert r.step(t) == o.step(t)
    for name, fid in (("prim", oracle_lib.FIELD_PRIM), ("dq", oracle_lib.FIELD_DQ),
                      ("flux_res", oracle_lib.FIELD_FLUX_RES), ("delun", oracle_lib.FIELD_DELUN)):
        assert np.array_equal(r.get(name), o.get(fid)), name
    ref_translated.TranslatedReference(c, p0, 0.8, 2.0)   # back to the defaults


_EXPLICIT_CHECK = """
import sys
sys.path.insert(0, {repo!r}); sys.path.insert(0, {pkg!r})
import numpy as np
from mfcfd import cloud
from oracle import ref_translated, oracle
for sup in (False, True):
    c = cloud.small_sphere(6, 100, r1=1.5)
    if sup:
        c = cloud.with_supersonic_boundary(c)
    p0 = cloud.initial_state(c, 0.8, 2.0)
    r = ref_translated.TranslatedReference(c, p0, 0.8, 2.0, libm="explicit")
    o = oracle.Oracle(c, 0.8, 2.0, update_variant=1)
    o.set_prim(p0)
    assert all(r.step(t) == o.step(t) for t in range(1, 5))
    for name, fid in (("prim", oracle.FIELD_PRIM), ("delup", oracle.FIELD_DELUP), ("delun", oracle.FIELD_DELUN)):
        assert np.array_equal(r.get(name), o.get(fid)), (sup, name)
print("ok")
"""


def test_oracle_explicit_update_matches_translated_reference(oracle_lib):
    """state_update.f90 (the reference's other state_update_mod), with and
    without supersonic points: restatement and reference agree bit for bit.
    Its own process: one translated build per process."""
    from oracle import ref_translated
    if not ref_translated.available("explicit"):
        pytest.skip("translated reference variant not built")
    code = _EXPLICIT_CHECK.format(repo=REPO, pkg=os.path.join(REPO, "3d-mfcfd_b200"))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stderr[-2000:]


_BACKUP_CHECK = """
import sys
sys.path.insert(0, {repo!r}); sys.path.insert(0, {pkg!r})
import numpy as np
from mfcfd import cloud
from oracle import ref_translated, oracle
for sup in (False, True):
    c = cloud.small_sphere(6, 100, r1=1.5)
    if sup:
        c = cloud.with_supersonic_boundary(c)
    p0 = cloud.initial_state(c, 0.8, 2.0)
    r = ref_translated.TranslatedReference(c, p0, 0.8, 2.0, libm="backup")
    o = oracle.Oracle(c, 0.8, 2.0, sweep_variant=1)
    o.set_prim(p0)
    for t in range(1, 4):
        a, b = r.step(t), o.step(t)
        assert np.array_equal(np.array(a).view(np.uint64), np.array(b).view(np.uint64)), (sup, t)
        for name, fid in (("prim", oracle.FIELD_PRIM), ("delup", oracle.FIELD_DELUP),
                          ("delun", oracle.FIELD_DELUN)):
            assert np.array_equal(r.get(name).view(np.uint64), o.get(fid).view(np.uint64)), (sup, t, name)
print("ok")
"""


def test_oracle_backup_sweeps_match_translated_reference(oracle_lib):
    """implicit_forward_and_reverse_sweeps_backup.f90 (the reference's other
    sweep driver: classes in index order, outer points swept with their own
    D_inv and L/U routines): restatement and reference agree bit for bit for
    three iterations, including where the driver breaks down (the outer
    D_inv's 1/delt operand is a tangential offset; the reference itself
    reaches NaN at outer points by the third iteration without supersonic
    points).  Its own process: one translated build per process."""
    from oracle import ref_translated
    if not ref_translated.available("backup"):
        pytest.skip("translated reference variant not built")
    code = _BACKUP_CHECK.format(repo=REPO, pkg=os.path.join(REPO, "3d-mfcfd_b200"))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stderr[-2000:]
