"""Host fit driver (ctpwa_minimize_box, the minimiser behind ctpwa_fit):
projected limited-memory BFGS with box bounds and fixed parameters, the
reference fit's scheme (example/fit.py:113-200: parameters clamped into their
bounds, gradient components pointing out of an active bound zeroed). No GPU."""
import ctypes

import numpy as np

from ctpwa_b200 import _lib

INF = float("inf")


def minimize(fun, x0, lo=None, hi=None, free=None, max_evals=500, history=20, ftol=1e-15, gtol=1e-10):
    lib = _lib.load()
    n = len(x0)
    x = np.ascontiguousarray(x0, dtype=np.float64).copy()
    lo = np.full(n, -INF) if lo is None else np.asarray(lo, dtype=np.float64)
    hi = np.full(n, INF) if hi is None else np.asarray(hi, dtype=np.float64)
    fr = np.ones(n, dtype=np.uint8) if free is None else np.asarray(free, dtype=np.uint8)
    calls = []

    def cb(xp, fp, gp, user):
        xv = np.ctypeslib.as_array(xp, shape=(n,)).copy()
        calls.append(xv)
        r = fun(xv)
        if isinstance(r, int):
            return r
        f, g = r
        fp[0] = f
        np.ctypeslib.as_array(gp, shape=(n,))[:] = g
        return 0

    fn = _lib.FG_FN(cb)
    out = np.zeros(4)
    dp = ctypes.POINTER(ctypes.c_double)
    rc = lib.ctpwa_minimize_box(fn, None, n, x.ctypes.data_as(dp), fr.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                                lo.ctypes.data_as(dp), hi.ctypes.data_as(dp), max_evals, history, ftol, gtol,
                                out.ctypes.data_as(dp))
    return rc, x, out, calls


def rosen(x):
    f = (1 - x[0]) ** 2 + 100 * (x[1] - x[0] ** 2) ** 2
    g = np.array([-2 * (1 - x[0]) - 400 * x[0] * (x[1] - x[0] ** 2), 200 * (x[1] - x[0] ** 2)])
    return f, g


def test_rosenbrock_unbounded():
    rc, x, out, calls = minimize(rosen, [-1.2, 1.0])
    assert rc == 0
    assert np.allclose(x, [1.0, 1.0], atol=1e-6), x
    assert out[0] < 1e-12 and out[1] == len(calls) <= 200 and out[3] in (0, 1)


def test_rosenbrock_with_active_bound():
    # x0 <= 0.5: the minimum sits on the bound at (0.5, 0.25), f = 0.25
    rc, x, out, calls = minimize(rosen, [-1.2, 1.0], hi=[0.5, INF])
    assert rc == 0
    assert np.allclose(x, [0.5, 0.25], atol=1e-7), x
    assert abs(out[0] - 0.25) < 1e-12
    assert all(c[0] <= 0.5 for c in calls)  # every evaluation inside the box


def test_bounded_quadratic_matches_clamped_minimum():
    rng = np.random.default_rng(4)
    n = 23
    a = rng.uniform(0.5, 50.0, n)
    c = rng.normal(0, 3, n)
    lo = np.where(rng.random(n) < 0.5, -1.0, -INF)
    hi = np.where(rng.random(n) < 0.5, 1.0, INF)
    q = rng.normal(0, 0.2, (n, n))
    M = np.diag(a) + q @ q.T  # coupled, positive definite

    def fun(x):
        d = x - c
        return float(d @ M @ d), 2 * M @ d

    rc, x, out, _ = minimize(fun, np.zeros(n), lo, hi)
    assert rc == 0 and out[3] in (0, 1)
    # KKT: projected gradient vanishes
    g = fun(x)[1]
    pg = np.clip(x - g, lo, hi) - x
    assert np.max(np.abs(pg)) < 1e-6 * np.max(np.abs(g) + 1)
    from scipy.optimize import minimize as sp_min

    ref = sp_min(fun, np.zeros(n), jac=True, method="L-BFGS-B",
                 bounds=[(None if l == -INF else l, None if h == INF else h) for l, h in zip(lo, hi)],
                 options={"ftol": 1e-15, "gtol": 1e-12, "maxfun": 5000})
    assert np.allclose(x, ref.x, atol=1e-6), np.max(np.abs(x - ref.x))


def test_fixed_parameters_stay_put():
    def fun(x):
        return float(np.sum((x - 3.0) ** 2)), 2 * (x - 3.0)

    x0 = np.array([1.0, 0.0, -2.0, 5.0])
    rc, x, out, calls = minimize(fun, x0, free=[0, 1, 1, 0])
    assert rc == 0
    assert x[0] == 1.0 and x[3] == 5.0
    assert np.allclose(x[1:3], 3.0, atol=1e-8)
    assert all(c[0] == 1.0 and c[3] == 5.0 for c in calls)


def test_start_outside_the_box_is_projected():
    def fun(x):
        return float(np.sum(x ** 2)), 2 * x

    rc, x, out, calls = minimize(fun, [5.0, 7.0], lo=[1.0, -INF], hi=[2.0, -3.0])
    assert rc == 0
    assert calls[0][0] == 2.0 and calls[0][1] == -3.0
    assert np.allclose(x, [1.0, -3.0])


def test_non_finite_trial_points_are_backtracked():
    # log barrier: f is +inf for x <= 0; minimum at x = 1
    def fun(x):
        if x[0] <= 0:
            return INF, np.array([0.0])
        return float(x[0] - np.log(x[0])), np.array([1 - 1 / x[0]])

    rc, x, out, _ = minimize(fun, [20.0])
    assert rc == 0 and abs(x[0] - 1.0) < 1e-6


def test_eval_budget_and_callback_error():
    rc, x, out, calls = minimize(rosen, [-1.2, 1.0], max_evals=7)
    assert rc == 0 and out[1] == len(calls) == 7 and out[3] == 2
    # the best point found is returned, never a rejected trial
    assert out[0] <= rosen(np.array([-1.2, 1.0]))[0]
    assert abs(out[0] - rosen(x)[0]) < 1e-15

    def bad(x):
        return 7

    rc, _, _, _ = minimize(bad, [0.0, 0.0])
    assert rc == 7


def test_argument_checks():
    lib = _lib.load()
    dp = ctypes.POINTER(ctypes.c_double)
    x = np.zeros(2)
    fr = np.ones(2, dtype=np.uint8)
    lo = np.array([1.0, 0.0])
    hi = np.array([0.0, 1.0])  # lo > hi
    out = np.zeros(4)
    fn = _lib.FG_FN(lambda *a: 0)
    rc = lib.ctpwa_minimize_box(fn, None, 2, x.ctypes.data_as(dp), fr.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                                lo.ctypes.data_as(dp), hi.ctypes.data_as(dp), 10, 5, 0.0, 0.0, out.ctypes.data_as(dp))
    assert rc != 0
