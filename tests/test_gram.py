"""Tensor-core Gram matrix of the phase-space sample against the FP64 oracle.

M_ab = (1/W) sum_e w_e sum_pol A_a conj(A_b) (the reference's normalisation
matrix, src/ComputeHessian.cu:1181-1197 with src/Analysis.cu:729-805). The
device forms the amplitudes in the mixed form (FP32) and the products on the
tensor cores (BF16 hi + lo operands, FP32 accumulation per 256-event tile, FP64
beyond); the oracle's amplitudes and sums are FP64. Tolerance: 1e-6 of the
largest |M_ab| elementwise (measured 3.5e-7 to 4.5e-7), and 1e-6 relative on the phase-space mean
intensity v^T M conj(v).
"""
import numpy as np
import pytest

from ctpwa_b200 import workloads
from oracle.binding import Oracle

pytestmark = pytest.mark.gpu

CASES = {"pipi_rho": 50_000, "pipi_3rho": 100_000, "kkpi": 200_000}


@pytest.mark.parametrize("name", list(CASES))
def test_gram_matches_oracle(tmp_path, name):
    import torch
    import ctpwa_b200

    cfg = workloads.make(name, tmp_path, n_phsp=CASES[name], n_data=2_000, n_bkg=0, accept_reject=False, seed=41)
    ana = ctpwa_b200.analysis(cfg)
    orc = Oracle(cfg)
    nV = ana.getNVector()
    p = workloads.true_params(nV, ana.getFreeResParams()[0].numpy())
    p[2 * nV:] *= 1 + 0.01 * np.random.default_rng(2).standard_normal(p.size - 2 * nV)
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    M = ana.getGram(pt).cpu().numpy()
    A = orc.columns(0, p[2 * nV:])  # [n, npol, nA] FP64
    R = np.einsum("epa,epb->ab", A, np.conj(A)) / A.shape[0]
    scale = np.max(np.abs(R))
    err = np.max(np.abs(M - R)) / scale
    assert err <= 1e-6, err
    # a second call at other parameters: no state carried over
    q = p.copy()
    q[2 * nV:] *= 1.01
    M2 = ana.getGram(torch.tensor(q, dtype=torch.float64, device="cuda")).cpu().numpy()
    A2 = orc.columns(0, q[2 * nV:])
    R2 = np.einsum("epa,epb->ab", A2, np.conj(A2)) / A2.shape[0]
    assert np.max(np.abs(M2 - R2)) <= 1e-6 * np.max(np.abs(R2))
    # the phase-space mean intensity as the quadratic form of the couplings
    _, _, parts = orc.nll_grad(p)
    cp = ana.getModel()["coupling"]
    v = np.array([r * complex(p[c], p[nV + c]) for c, r in zip(cp["amp_chain"], cp["ratio"])])
    f = np.real(v @ M @ np.conj(v))
    mean = parts[2]  # the phase-space factor: weighted intensity sum / weight total
    assert abs(f - mean) <= 1e-6 * abs(mean), (f, mean)


HESS_CASES = {"pipi_rho": (100_000, 10_000, 0), "pipi_3rho": (200_000, 20_000, 2_000), "kkpi": (300_000, 30_000, 3_000)}


@pytest.mark.parametrize("name", list(HESS_CASES))
def test_gram_hessian_matches_exact(tmp_path, name):
    """getHessian(method="gram"): the coupling block from tensor-core Gram
    sums (sum (w/f) A conj(A), sum (w/f^2) c conj(c) over data and background,
    the normalisation matrix over phase space), the resonance rows exact,
    against the exact FP64 Hessian: 2e-5 of the largest entry over the whole
    matrix (the coupling block carries the Gram's ~4e-7 rounding, amplified
    by the cancellation between the data and normalisation terms)."""
    import torch
    import ctpwa_b200

    nph, nda, nbk = HESS_CASES[name]
    cfg = workloads.make(name, tmp_path, n_phsp=nph, n_data=nda, n_bkg=nbk, accept_reject=False, seed=43)
    ana = ctpwa_b200.analysis(cfg)
    nV = ana.getNVector()
    p = workloads.true_params(nV, ana.getFreeResParams()[0].numpy())
    p[2 * nV:] *= 1 + 0.01 * np.random.default_rng(5).standard_normal(p.size - 2 * nV)
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    He = ana.getHessian(pt, "exact").cpu().numpy()
    Hg = ana.getHessian(pt, "gram").cpu().numpy()
    scale = np.max(np.abs(He))
    err = np.max(np.abs(Hg - He)) / scale
    assert err <= 2e-5, err
    # the resonance rows are the exact ones
    n2 = 2 * nV
    assert np.max(np.abs(Hg[n2:] - He[n2:])) <= 1e-9 * scale
    assert np.array_equal(Hg, Hg.T)
