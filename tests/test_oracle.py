"""Pins the CPU oracle: against the reference's own math compiled from its
sources (oracle/_ref, built by `make -C oracle ref` where the reference tree
exists), against analytic identities, and its gradient against central
finite differences."""
import ctypes

import numpy as np
import pytest

from ctpwa_b200 import toymc, workloads
from oracle.binding import Oracle, oracle_lib, ptr, ref_lib

_I = ctypes.POINTER(ctypes.c_int)


def _boosted_events(n, seed):
    p4 = toymc.phase_space(3.0969, (0.493677, 0.493677, 0.13495), n, seed)
    rng = np.random.default_rng(seed)
    out = []
    for e in range(n):
        beta = rng.uniform(-0.5, 0.5, 3)
        out.append(toymc._boost(p4[e], np.tile(beta, (3, 1))))
    return out


VERTICES = [(3, 3, 1, 3, 1), (3, 5, 1, 5, 2), (3, 1, 1, 1, 1), (5, 1, 1, 1, 2), (3, 3, 3, 3, 0), (3, 3, 3, 5, 2),
            (3, 2, 2, 1, 1), (4, 3, 2, 4, 2), (3, 1, 3, 3, 1), (5, 3, 3, 3, 2), (2, 2, 1, 2, 1), (7, 3, 1, 3, 3)]


@pytest.fixture(scope="module")
def ref():
    r = ref_lib()
    if r is None:
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    return r


@pytest.mark.parametrize("v", VERTICES)
def test_vertex_tensor_matches_reference(ref, v):
    dj, dj1, dj2, S, L = v
    orc = oracle_lib()
    n = dj * dj1 * dj2
    for q in _boosted_events(40, 7 + dj + 3 * L):
        a = np.ascontiguousarray(q[0])
        b = np.ascontiguousarray(q[1] + q[2] if dj2 == 1 else q[1])
        o1, o2 = np.zeros(2 * n), np.zeros(2 * n)
        orc.orc_pwa_amp(ptr(a), dj1, ptr(b), dj2, dj, S, L, ptr(o1))
        ref.ref_pwa_amp(ptr(a), dj1, ptr(b), dj2, dj, S, L, ptr(o2))
        assert np.max(np.abs(o1 - o2)) <= 1e-13 * max(1.0, np.max(np.abs(o2)))


def test_clebsch_matches_reference_and_is_orthonormal(ref):
    orc = oracle_lib()
    for dj1 in range(1, 6):
        for dj2 in range(1, 6):
            for dJ in range(abs(dj1 - dj2) + 1, dj1 + dj2, 2):
                for m1 in range(-(dj1 - 1), dj1, 2):
                    for m2 in range(-(dj2 - 1), dj2, 2):
                        a = orc.orc_clebsch(dj1, m1, dj2, m2, dJ, m1 + m2)
                        assert a == pytest.approx(ref.ref_clebsch(dj1, m1, dj2, m2, dJ, m1 + m2), abs=1e-14)
            # orthonormality: sum_{m1,m2} <..|J M><..|J' M> = delta_JJ'
            for dJ in range(abs(dj1 - dj2) + 1, dj1 + dj2, 2):
                for M in range(-(dJ - 1), dJ, 2):
                    s = sum(orc.orc_clebsch(dj1, m1, dj2, M - m1, dJ, M) ** 2 for m1 in range(-(dj1 - 1), dj1, 2))
                    assert s == pytest.approx(1.0, abs=1e-12)


def _q(m, a, b):
    v = (m * m - (a + b) ** 2) * (m * m - (a - b) ** 2)
    return np.sqrt(max(v, 0.0)) / (2 * m)


MODELS = [(0, [0.8955, 0.047], [], 1), (0, [1.4256, 0.0985], [], 2), (1, [0.775, 0.149], [], 1), (2, [1.2], [], 1),
          (3, [0.99, 0.2, 0.4], [0.1396, 0.1396, 0.4937, 0.4937], 0), (6, [0.775, 0.149], [0.1396, 0.1396], 1)]


@pytest.mark.parametrize("case", MODELS)
def test_lineshapes_match_reference_symbolic_path(ref, case):
    t, par, ch, Lmin = case
    orc = oracle_lib()
    P, nch = len(par), len(ch) // 2
    m1, m2 = (0.1396, 0.1396) if t == 6 else (0.493677, 0.13495)
    mdep = np.zeros(2, dtype=np.int32)
    mfix = np.array([m1, m2])
    cha = np.array(ch if ch else [0.0])
    para = np.array(par, dtype=float)
    h = ref.ref_model_build(t, 1, Lmin, 3.0, P, nch, ptr(cha), mdep.ctypes.data_as(_I), ptr(mfix), 1)
    rng = np.random.default_rng(t)
    z8 = np.zeros(8)
    for i in range(100):
        m = rng.uniform(m1 + m2 + 1e-3, 2.5)
        q = _q(m, m1, m2)
        L = Lmin + i % 2
        o1, o2 = np.zeros(2 + 2 * P), np.zeros(2 + 2 * P + 2 * P * P)
        orc.orc_model_eval(t, Lmin, 3.0, P, nch, ptr(cha), mdep.ctypes.data_as(_I), ptr(mfix), 1, ptr(para), m, q, L,
                           3.0, m1, m2, ptr(o1))
        ref.ref_aux_eval(h, ptr(para), P, m, q, L, 3.0, m1, m2, ptr(z8), ptr(o2))
        assert np.max(np.abs(o1[:2] - o2[:2])) <= 1e-13 * np.max(np.abs(o2[:2]))
        assert np.max(np.abs(o1[2:] - o2[2:2 + 2 * P])) <= 1e-12 * max(1e-300, np.max(np.abs(o2[2:2 + 2 * P])))
    ref.ref_aux_free(h)


EXPRS = [("Flatte(mass, gKK, gpipi, 0.493677, 0.493677, 0.13957, 0.13957) * Bf(1, q, q0, 3.0)", "mass,gKK,gpipi",
          [1.68, 0.3, 0.1]),
         ("p0^2/(p0^2 - m^2 - 1j*p0*p1)", "p0,p1", [1.66, 0.125]),
         ("BWR(p0, p1, 1, 3.0) * Bf(1, q, q0(m), 3.0)", "p0,p1", [1.66, 0.125]),
         ("exp(1j*p2)*BW(p0,p1) + sqrt(m - p0) - log(m*p1) + sin(p2)*cos(m) + abs(p1-1j)/conj(p0+1j) + Re(p0*1j)"
          " - Im(p1) + csqrt(-m) + q0", "p0,p1,p2", [1.2, 0.2, 0.3]),
         ("-p0^2^0.5 + (m/p1)^(1j*p1) - -p1", "p0,p1", [1.4, 0.3]),
         # the reference's constant folding and IEEE signed zeros on the branch cut of log / pow
         ("(-m)^0.5 * (m*-2)^p2 + log(-p1*m) + exp(-m)*(-1)^p2", "p0,p1,p2", [1.68, 0.3, 0.1]),
         ("(-p0 - m)^1.5 + conj(-m)^0.3 - (m/-1)^0.5 + (-1*m)^0.5 + sin(-p0)^2.5 * cos(p0)^0.5", "p0,p1",
          [1.68, 0.3]),
         ("0^(m-2) + p0^1*p1^1 + 1^m + (0-m)^0.5 - -(-m)^0.5 + 0*log(0*m) + (-(m^2-p0^2))^p1", "p0,p1",
          [1.68, 0.3])]

# folded constants that the reference evaluates to NaN (real pow of a negative number)
NAN_EXPRS = ["(-2)^0.5 + p0", "(m*0-1)^0.5 * p0"]


@pytest.mark.parametrize("case", EXPRS)
def test_custom_expressions_match_reference(ref, case):
    e, names, par = case
    orc = oracle_lib()
    P = len(par)
    para = np.array(par, dtype=float)
    h = ref.ref_custom_build(e.encode(), names.encode())
    assert h
    rng = np.random.default_rng(P)
    z8 = np.zeros(8)
    for i in range(100):
        m = rng.uniform(1.0, 2.5)
        q = _q(m, 0.493677, 0.493677)
        o1, o2 = np.zeros(2 + 2 * P), np.zeros(2 + 2 * P + 2 * P * P)
        err = ctypes.create_string_buffer(256)
        assert orc.orc_custom_eval(e.encode(), names.encode(), ptr(para), P, m, q, 1, 3.0, 0.493677, 0.493677,
                                   ptr(o1), err, 256) == 0
        ref.ref_aux_eval(h, ptr(para), P, m, q, 1, 3.0, 0.493677, 0.493677, ptr(z8), ptr(o2))
        assert np.max(np.abs(o1[:2] - o2[:2])) <= 1e-13 * np.max(np.abs(o2[:2]))
        assert np.max(np.abs(o1[2:] - o2[2:2 + 2 * P])) <= 1e-12 * max(1e-300, np.max(np.abs(o2[2:2 + 2 * P])))
    ref.ref_aux_free(h)


@pytest.mark.parametrize("expr", NAN_EXPRS)
def test_custom_expression_nan_folding_matches_reference(ref, expr):
    orc = oracle_lib()
    para = np.array([1.5])
    h = ref.ref_custom_build(expr.encode(), b"p0")
    assert h
    o1, o2 = np.zeros(4), np.zeros(6)
    err = ctypes.create_string_buffer(256)
    m = 1.3
    q = _q(m, 0.493677, 0.493677)
    assert orc.orc_custom_eval(expr.encode(), b"p0", ptr(para), 1, m, q, 1, 3.0, 0.493677, 0.493677, ptr(o1),
                               err, 256) == 0
    ref.ref_aux_eval(h, ptr(para), 1, m, q, 1, 3.0, 0.493677, 0.493677, ptr(np.zeros(8)), ptr(o2))
    assert np.isnan(o2[0]) and np.isnan(o1[0])
    ref.ref_aux_free(h)


def test_wigner_small_d_is_orthogonal():
    """d^j(beta) is a real orthogonal matrix for every j <= 3 (analytic
    known answer): sum_m d^j_{m1 m}(b) d^j_{m2 m}(b) = delta_{m1 m2}, and
    d^j(0) = 1."""
    orc = oracle_lib()
    for dim in range(1, 8):
        ms = list(range(dim - 1, -dim, -2))
        for beta in (0.0, 0.37, 1.2, 2.9):
            d = np.array([[orc.orc_small_d(dim, a, b, beta) for b in ms] for a in ms])
            assert np.max(np.abs(d @ d.T - np.eye(dim))) <= 1e-13, (dim, beta)
            if beta == 0.0:
                assert np.max(np.abs(d - np.eye(dim))) <= 1e-15


def test_spherical_harmonics_are_orthonormal():
    """Y_l^m orthonormal on the sphere for l <= 4 (analytic known answer),
    by Gauss-Legendre quadrature in cos(theta) and the trapezoid rule in phi
    (exact for these polynomials and trigonometric terms)."""
    orc = oracle_lib()
    x, wx = np.polynomial.legendre.leggauss(24)
    nphi = 24
    phis = 2 * np.pi * np.arange(nphi) / nphi
    lm = [(l, m) for l in range(5) for m in range(-l, l + 1)]
    Y = np.zeros((len(lm), x.size, nphi), dtype=complex)
    out = np.zeros(2)
    for i, (l, m) in enumerate(lm):
        for a, c in enumerate(x):
            for b, ph in enumerate(phis):
                orc.orc_ylm(l, m, float(np.arccos(c)), float(ph), ptr(out))
                Y[i, a, b] = out[0] + 1j * out[1]
    w = wx[:, None] * (2 * np.pi / nphi)
    G = np.einsum("iab,jab,ab->ij", np.conj(Y), Y, np.broadcast_to(w, Y.shape[1:]))
    assert np.max(np.abs(G - np.eye(len(lm)))) <= 1e-12


def test_barrier_and_breit_wigner_identities():
    """Bf(L, q0, q0) = 1 and |BWR(m0)| = 1/(m0 G0) (analytic known answers)."""
    orc = oracle_lib()
    mdep = np.zeros(2, dtype=np.int32)
    mfix = np.array([0.493677, 0.13495])
    cha = np.array([0.0])
    for m0, g0, L in [(0.8955, 0.047, 1), (1.4256, 0.0985, 2)]:
        q0 = _q(m0, *mfix)
        o = np.zeros(6)
        para = np.array([m0, g0])
        orc.orc_model_eval(0, L, 3.0, 2, 0, ptr(cha), mdep.ctypes.data_as(_I), ptr(mfix), 1, ptr(para), m0, q0, L, 3.0,
                           mfix[0], mfix[1], ptr(o))
        assert np.hypot(o[0], o[1]) == pytest.approx(1.0 / (m0 * g0), rel=1e-12)


@pytest.mark.parametrize("name", ["pipi_rho", "pipi_3rho", "kkpi"])
def test_oracle_gradient_matches_finite_differences(tmp_path, name):
    cfg = workloads.make(name, tmp_path, n_phsp=3000, n_data=800, n_bkg=200 if name != "pipi_rho" else 0,
                         accept_reject=False, seed=2)
    o = Oracle(cfg)
    rng = np.random.default_rng(4)
    theta = workloads.SIZES  # noqa: F841 (sizes only documented)
    m = __import__("ctpwa_b200").describe(cfg)
    p = workloads.true_params(o.nV, [s["init"] for s in m["slots"]])
    p[2 * o.nV:] *= 1 + 0.01 * rng.standard_normal(o.nT)
    f, g, _ = o.nll_grad(p)
    fd = np.zeros_like(g)
    for i in range(p.size):
        h = 1e-6 * max(1.0, abs(p[i]))
        q = p.copy()
        q[i] += h
        fp = o.nll_grad(q)[0]
        q[i] -= 2 * h
        fm = o.nll_grad(q)[0]
        fd[i] = (fp - fm) / (2 * h)
    assert np.max(np.abs(fd - g)) <= 1e-6 * np.max(np.abs(g))


def test_nll_invariant_under_global_coupling_scale(tmp_path):
    """The NLL is invariant under v -> c v (data and normalisation scale alike)."""
    cfg = workloads.make("kkpi", tmp_path, n_phsp=2000, n_data=500, n_bkg=0, accept_reject=False, seed=5)
    o = Oracle(cfg)
    m = __import__("ctpwa_b200").describe(cfg)
    p = workloads.true_params(o.nV, [s["init"] for s in m["slots"]])
    f1 = o.nll_grad(p)[0]
    q = p.copy()
    q[:2 * o.nV] *= 3.7
    assert o.nll_grad(q)[0] == pytest.approx(f1, rel=1e-12)
