"""Fit-level precision of the mixed form against the plain FP64 path.

J/psi -> pi+ pi- pi0 with three rho chains (rho(770), rho(1450), rho(1700)
each), 500k data events by accept-reject, 5M phase space and 50k background
(weight 0.8). From 20 seeded starting points around the generating
parameters
the library's fit driver minimises the NLL once in FP64 and once in the
mixed form. Both fits must reach the same minimum (NLL within 0.01) and
every fitted parameter must agree within 0.01 sigma, sigma from
the inverse of the exact FP64 Hessian at the FP64 minimum (example/fit.py:
213, 333 form the errors the same way).
"""
import numpy as np
import pytest

from ctpwa_b200 import workloads

pytestmark = pytest.mark.gpu


def start_point(p_true, nV, res, seed):
    """The generating parameters moved at random: couplings by 20 % (the
    first one stays fixed to 1 + 0i), resonance parameters by up to 2 % of
    their allowed range, seeded, so that every start lies in the basin of
    the generating minimum (the model has other local minima, which would
    compare the optimiser's paths rather than the precision of the minimum)."""
    rng = np.random.default_rng(seed)
    p = p_true.copy()
    for i in range(1, nV):
        p[i] *= 1 + 0.2 * rng.standard_normal()
        p[nV + i] *= 1 + 0.2 * rng.standard_normal()
    lo, hi = res[1], res[2]
    th = p[2 * nV:] + (rng.uniform(size=res.shape[1]) - 0.5) * 0.04 * (hi - lo)
    p[2 * nV:] = np.clip(th, lo + 1e-7 * (hi - lo), hi - 1e-7 * (hi - lo))
    return p


def test_mixed_fits_within_a_hundredth_of_sigma(tmp_path):
    import torch
    import ctpwa_b200

    cfg = workloads.make("pipi_3rho", tmp_path, n_phsp=5_000_000, n_data=500_000, n_bkg=50_000, bkg_weight=0.8,
                         seed=23)
    ana = ctpwa_b200.analysis(cfg)
    nV, nP = ana.getNVector(), ana.getNParams()
    res = ana.getFreeResParams().numpy()
    p_true = workloads.true_params(nV, res[0])
    free = np.ones(nP, dtype=bool)
    free[0] = free[nV] = False
    worst = 0.0
    for k in range(20):
        x0 = start_point(p_true, nV, res, 1000 + k)
        x64, n64, _, _, s64, _ = ana.fit(x0, max_evals=3000, ftol=1e-15, gtol=1e-8, precision="fp64")
        xmx, nmx, _, _, smx, _ = ana.fit(x0, max_evals=3000, ftol=1e-15, gtol=1e-8, precision="mixed")
        # status 3 (no decrease along the search direction) ends a fit whose
        # remaining decrease is below the NLL's rounding: it is converged
        assert s64 in (0, 1, 3) and smx in (0, 1, 3), (k, s64, smx)
        assert abs(nmx - n64) < 1e-2, (k, n64, nmx)
        pt = torch.tensor(x64, dtype=torch.float64, device="cuda")
        C = ana.getCovariance(pt, free=free).cpu().numpy()
        sigma = np.sqrt(np.diag(C)[free])
        d = np.abs(xmx[free] - x64[free]) / sigma
        worst = max(worst, float(d.max()))
        assert d.max() < 0.01, (k, d.max(), s64, smx, n64, nmx)
