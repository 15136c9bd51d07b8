"""The solver's own exp/log/erf (3d-mfcfd_b200/csrc/mfmath.h), host build.

Accuracy against 40-digit mpmath on seeded samples, and agreement with
glibc (which the Fortran reference calls) on most arguments.  The GPU build
of the same functions is checked bit for bit through the parity tests.
"""
import math

import numpy as np
import pytest

mp = pytest.importorskip("mpmath")
mp.mp.dps = 40


def _ulp_err(y, x, f):
    out = []
    for a, v in zip(y, x):
        r = f(mp.mpf(float(v)))
        rf = float(r)
        if rf == 0.0:
            out.append(0.0 if a == 0.0 else np.inf)
            continue
        out.append(float(abs(mp.mpf(float(a)) - r) / math.ulp(rf)))
    return np.array(out)


CASES = {
    "exp": (lambda rng: np.concatenate([rng.uniform(-5, 5, 800), rng.uniform(-700, 700, 300),
                                        rng.uniform(-40, 0, 300)]), mp.exp, 0.6),
    "log": (lambda rng: np.concatenate([rng.uniform(0.05, 5, 800), np.exp(rng.uniform(-60, 60, 300)),
                                        1 + rng.uniform(-1e-3, 1e-3, 300)]), mp.log, 0.6),
    "erf": (lambda rng: np.concatenate([rng.uniform(-1, 1, 800), rng.uniform(-6.5, 6.5, 600),
                                        rng.uniform(-1e-6, 1e-6, 100)]), mp.erf, 0.8),
}


@pytest.mark.parametrize("fn", sorted(CASES))
def test_accuracy(oracle_lib, fn):
    gen, f, bound = CASES[fn]
    x = gen(np.random.default_rng(1234))
    y = oracle_lib.libm_eval(fn, 1, x)
    err = _ulp_err(y, x, f)
    assert err.max() < bound, (fn, err.max())
    g = oracle_lib.libm_eval(fn, 0, x)
    assert np.mean(y == g) > 0.9     # mostly bitwise equal to glibc


def test_special_values(oracle_lib):
    x = np.array([0.0, -0.0, 1.0, -1.0, 6.0, -6.0, 30.0, np.inf, -np.inf])
    e = oracle_lib.libm_eval("erf", 1, x)
    assert e[0] == 0.0 and e[4] == 1.0 and e[5] == -1.0 and e[6] == 1.0
    assert e[7] == 1.0 and e[8] == -1.0
    assert np.all(oracle_lib.libm_eval("erf", 1, -x[2:6]) == -e[2:6])
    ex = oracle_lib.libm_eval("exp", 1, np.array([0.0, -800.0, 800.0, 1.0]))
    assert ex[0] == 1.0 and ex[1] == 0.0 and ex[2] == np.inf
    assert ex[3] == math.e
    lg = oracle_lib.libm_eval("log", 1, np.array([1.0, 0.0, -1.0, 2.0, 5e-320]))
    assert lg[0] == 0.0 and lg[1] == -np.inf and np.isnan(lg[2]) and lg[3] == math.log(2.0)
    assert abs(lg[4] - math.log(5e-320)) <= 2 * math.ulp(math.log(5e-320))
