"""The identities the normalisation cache rests on, on the oracle's FP64
amplitudes (CPU; the device kernels are checked against the oracle in
tests/test_norm_cache.py).

With A[e, p, a] the amplitude of column a in polarisation p of phase-space
event e, S[e, p] = sum_a v_a A[e, p, a] and f_e = sum_p |S[e, p]|^2:
  sum_e f_e                      = sum_ab v_a conj(v_b) M[a, b],   M = sum_e,p A_a conj(A_b)
  sum_e,p conj(A[e, p, a]) S[e, p] = sum_b conj(M[a, b]) v_b          (coupling-gradient sums)
  d/dtheta_j sum_e f_e           = 2 Re sum_ab v_a conj(v_b) D_j[a, b],  D_j = sum_e,p dA_a/dtheta_j conj(A_b)
the matrices of the reference's phase-space quadratic form
(src/Analysis.cu:748-829, src/ComputeNLL.cu:575-597) and their
resonance-parameter derivatives.
"""
import numpy as np

import ctpwa_b200
from ctpwa_b200 import workloads
from oracle.binding import Oracle


def test_quadratic_form_identities_on_oracle_amplitudes(tmp_path):
    cfg = workloads.make("pipi_3rho", tmp_path, n_phsp=3_000, n_data=300, n_bkg=0, accept_reject=False, seed=3,
                         gpu_generator=False)
    orc = Oracle(cfg)
    nV, nT = orc.nV, orc.nT
    th = orc.theta_init()[0]
    p = workloads.true_params(nV, th)
    cp = ctpwa_b200.describe(cfg)["coupling"]
    v = np.array([r * complex(p[c], p[nV + c]) for c, r in zip(cp["amp_chain"], cp["ratio"])])

    A = orc.columns(0, th)  # [n, npol, nA]
    M = np.einsum("epa,epb->ab", A, np.conj(A))
    S = np.einsum("epa,a->ep", A, v)
    f = np.sum(np.abs(S) ** 2, axis=1)
    # the intensity sum as the quadratic form, and the oracle's phase-space factor
    fq = np.real(v @ M @ np.conj(v))
    assert abs(f.sum() - fq) <= 1e-12 * f.sum()
    _, _, parts = orc.nll_grad(p)
    assert abs(parts[2] - f.sum() / A.shape[0]) <= 1e-12 * parts[2]
    # coupling-gradient sums
    g_direct = np.einsum("epa,ep->a", np.conj(A), S)
    g_quad = np.conj(M) @ v
    assert np.max(np.abs(g_direct - g_quad)) <= 1e-12 * np.max(np.abs(g_direct))
    # resonance-parameter derivative of the intensity sum from D_j (central
    # differences of the oracle's amplitudes and of the intensity sum)
    for j in range(nT):
        h = 1e-6 * max(abs(th[j]), 1e-2)
        tp, tm = th.copy(), th.copy()
        tp[j] += h
        tm[j] -= h
        Ap, Am = orc.columns(0, tp), orc.columns(0, tm)
        dA = (Ap - Am) / (2 * h)
        D = np.einsum("epa,epb->ab", dA, np.conj(A))
        dq = 2.0 * np.real(v @ D @ np.conj(v))
        fp = np.sum(np.abs(np.einsum("epa,a->ep", Ap, v)) ** 2)
        fm = np.sum(np.abs(np.einsum("epa,a->ep", Am, v)) ** 2)
        dfd = (fp - fm) / (2 * h)
        assert abs(dq - dfd) <= 1e-6 * max(abs(dfd), 1e-3 * f.sum()), (j, dq, dfd)
