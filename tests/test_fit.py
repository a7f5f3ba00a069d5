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


# ---------------------------------------------------------------------------
# Newton fit (ctpwa_minimize_box_newton, the minimiser behind ctpwa_fit_newton)
# ---------------------------------------------------------------------------
def newton(fun, hess, x0, lo=None, hi=None, free=None, max_iter=100, xtol=1e-10, gtol=1e-12, fnoise=0.0):
    lib = _lib.load()
    n = len(x0)
    x = np.ascontiguousarray(x0, dtype=np.float64).copy()
    lo = np.full(n, -INF) if lo is None else np.asarray(lo, dtype=np.float64)
    hi = np.full(n, INF) if hi is None else np.asarray(hi, dtype=np.float64)
    fr = np.ones(n, dtype=np.uint8) if free is None else np.asarray(free, dtype=np.uint8)
    calls = {"f": 0, "h": 0}

    def cb(xp, fp, gp, user):
        calls["f"] += 1
        r = fun(np.ctypeslib.as_array(xp, shape=(n,)).copy())
        if isinstance(r, int):
            return r
        fp[0] = r[0]
        np.ctypeslib.as_array(gp, shape=(n,))[:] = r[1]
        return 0

    def hb(xp, hp, user):
        calls["h"] += 1
        r = hess(np.ctypeslib.as_array(xp, shape=(n,)).copy())
        if isinstance(r, int):
            return r
        np.ctypeslib.as_array(hp, shape=(n * n,))[:] = np.asarray(r, dtype=np.float64).reshape(-1)
        return 0

    fn, hn = _lib.FG_FN(cb), _lib.HESS_FN(hb)
    out = np.zeros(4)
    dp = ctypes.POINTER(ctypes.c_double)
    rc = lib.ctpwa_minimize_box_newton(fn, hn, None, n, x.ctypes.data_as(dp),
                                       fr.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), lo.ctypes.data_as(dp),
                                       hi.ctypes.data_as(dp), max_iter, xtol, gtol, fnoise, out.ctypes.data_as(dp))
    return rc, x, out, calls


def rosen_hess(x):
    return np.array([[2 - 400 * (x[1] - 3 * x[0] ** 2), -400 * x[0]], [-400 * x[0], 200.0]])


def test_newton_rosenbrock_unbounded():
    # the start's Hessian is indefinite: damped steps until it is not
    rc, x, out, calls = newton(rosen, rosen_hess, [-1.2, 1.0])
    assert rc == 0 and out[3] in (0, 1), out
    assert np.allclose(x, [1.0, 1.0], atol=1e-9), x
    assert out[2] == calls["h"] <= 60 and out[1] == calls["f"]


def test_newton_active_bound_and_fixed_parameter():
    rc, x, out, _ = newton(rosen, rosen_hess, [-1.2, 1.0], hi=[0.5, INF])
    assert rc == 0 and np.allclose(x, [0.5, 0.25], atol=1e-9), (x, out)
    # x1 fixed at 0.64: minimum over x0 alone (x0 = 0.8 solves x1 = x0^2 and x0 ~ 1)
    rc, x, out, _ = newton(rosen, rosen_hess, [0.3, 0.64], free=[1, 0])
    assert rc == 0 and x[1] == 0.64
    g = rosen(x)[1]
    assert abs(g[0]) < 1e-8, (x, g)


def test_newton_stays_in_the_basin_of_a_singular_well():
    # a quadratic bowl at 1 plus a log well at 2.5 that goes to -inf (the
    # shape a subtracted background event gives a likelihood): from inside
    # the bowl's basin the iteration converges to the bowl's minimum
    a, w = 2.5, 0.8

    def fun(x):
        d = x[0] - a
        return 50 * (x[0] - 1) ** 2 + w * np.log(d * d), np.array([100 * (x[0] - 1) + 2 * w / d])

    def hess(x):
        d = x[0] - a
        return np.array([[100 - 2 * w / (d * d)]])

    rc, x, out, _ = newton(fun, hess, [0.6])
    assert rc == 0 and out[3] in (0, 1)
    assert abs(fun(x)[1][0]) < 1e-9 and abs(x[0] - 1) < 0.02 and hess(x)[0, 0] > 0


def test_newton_tolerates_rounding_noise_of_f():
    # f carries a deterministic perturbation of 1e-6: steps whose predicted
    # decrease is below fnoise are kept, and the iteration ends on the step
    # size instead of failing to find a decrease
    def fun(x):
        f, g = rosen(x)
        return f + 1e-6 * np.sin(1e7 * x[0] + 3e7 * x[1]), g

    rc, x, out, _ = newton(fun, rosen_hess, [0.8, 0.7], xtol=1e-8, fnoise=1e-5)
    assert rc == 0 and out[3] == 1, out
    assert np.allclose(x, [1.0, 1.0], atol=1e-7), x


def test_newton_callback_errors_and_arguments():
    rc, _, _, _ = newton(lambda x: 7, rosen_hess, [0.0, 0.0])
    assert rc == 7
    rc, _, _, _ = newton(rosen, lambda x: 9, [0.0, 0.0])
    assert rc == 9
    rc, _, _, _ = newton(rosen, rosen_hess, [0.0, 0.0], lo=[1.0, -INF], hi=[0.0, INF])
    assert rc != 0
    rc, _, _, _ = newton(rosen, rosen_hess, [0.0, 0.0], max_iter=0)
    assert rc != 0
