"""Accuracy of the deterministic elementary functions shared by the GPU kernels
and the oracle (double-evaluated, rounded once to float), against float64/
long-double references: correctly rounded in all but a handful of cases."""
import numpy as np
import pytest


def _ulp_err(got, ref):
    got = np.asarray(got, np.float32)
    ref64 = np.asarray(ref, np.float64)
    rf = ref64.astype(np.float32)
    sp = np.spacing(np.abs(rf).astype(np.float32)).astype(np.float64)
    sp[sp == 0] = np.finfo(np.float32).tiny
    return np.abs(got.astype(np.float64) - ref64) / sp


CASES = [
    (0, "sin", lambda a, b: np.sin(a), lambda r: (r.uniform(-50, 50, 400000), None)),
    (1, "cos", lambda a, b: np.cos(a), lambda r: (r.uniform(-50, 50, 400000), None)),
    (2, "tan", lambda a, b: np.tan(a), lambda r: (r.uniform(-1.5, 1.5, 400000), None)),
    (3, "exp", lambda a, b: np.exp(a), lambda r: (r.uniform(-100, 88, 400000), None)),
    (4, "log", lambda a, b: np.log(a), lambda r: (np.exp(r.uniform(-85, 85, 400000)), None)),
    (5, "pow", lambda a, b: np.power(a, b), lambda r: (r.uniform(0.001, 3, 400000), r.uniform(-10, 10, 400000))),
    (6, "atan2", lambda a, b: np.arctan2(a, b), lambda r: (r.normal(size=400000), r.normal(size=400000))),
    (7, "acos", lambda a, b: np.arccos(a), lambda r: (r.uniform(-1, 1, 400000), None)),
]


@pytest.mark.parametrize("fn,name,ref,gen", CASES)
def test_portable_math_correctly_rounded(oracle_mod, fn, name, ref, gen):
    orc = oracle_mod.Oracle(libm=False)
    rng = np.random.default_rng(fn)
    a, b = gen(rng)
    a = a.astype(np.float32)
    b = None if b is None else b.astype(np.float32)
    got = orc.math_eval(fn, a, b)
    with np.errstate(all="ignore"):
        r = ref(np.longdouble(a) if b is None else np.longdouble(a), None if b is None else np.longdouble(b))
    err = _ulp_err(got, r)
    fin = np.isfinite(np.asarray(r, np.float64)) & (np.abs(np.asarray(r, np.float64)) < 3e38)
    assert err[fin].max() <= 1.0, f"{name}: max {err[fin].max()} ulp"
    assert np.mean(err[fin] <= 0.5 + 1e-6) > 0.9999, f"{name}: {np.mean(err[fin] > 0.5)} not correctly rounded"


def test_special_values(oracle_mod):
    orc = oracle_mod.Oracle(libm=False)
    inf, nan = np.float32(np.inf), np.float32(np.nan)
    f = lambda fn, a, b=None: orc.math_eval(fn, np.array([a], np.float32), None if b is None else np.array([b], np.float32))[0]  # noqa
    assert np.isnan(f(0, inf)) and np.isnan(f(1, nan)) and f(3, -200.0) == 0.0 and f(3, 100.0) == inf
    assert f(4, 0.0) == -inf and np.isnan(f(4, -1.0)) and f(5, 0.0, 5.0) == 0.0 and f(5, 2.0, 0.0) == 1.0
    assert np.signbit(f(0, -0.0)) and f(6, 0.0, -1.0) == np.float32(np.pi) and f(7, 1.0) == 0.0
    assert f(5, -2.0, 3.0) == -8.0 and np.isnan(f(5, -2.0, 0.5))
