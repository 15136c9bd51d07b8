"""Rebuild the translated reference from the reference sources (where the
checkout exists) and check it still produces the committed fixtures."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

REF = "/root/reference"
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "sphere_600.npz")

pytestmark = pytest.mark.skipif(not os.path.isdir(REF), reason="reference checkout absent")


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
