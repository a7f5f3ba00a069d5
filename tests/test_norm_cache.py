"""Normalisation cache: evaluations at fixed resonance parameters from FP64
quadratic forms in the couplings instead of the phase-space pass.

The reference keeps its phase-space matrix A^H diag(w/W) A between
evaluations when no resonance parameter is free (src/Analysis.cu:748-829,
quadratic form src/ComputeNLL.cu:575-597). The cache holds that matrix in
FP64 plus the matrices of the lineshape derivatives, so the whole gradient
follows as well. Checks, on the same seeded inputs:
  - cached FP64 NLL and gradient equal the full FP64 pass and the oracle
    (1e-10 relative on the NLL, 1e-9 of the largest gradient component),
    at the build point and at other couplings with the same resonance
    parameters; the mixed form from the cache stays within its 1e-3 budget;
  - weighted phase space (per-event weight files): the weighted matrix for
    the coupling gradient, the unweighted one for the intensity sum;
  - other resonance parameters through the cached entry point are flagged
    invalid (NLL 1e30, zero gradient); the host entry point falls back to
    the full pass for them;
  - a fit with every resonance parameter fixed builds the cache itself and
    ends where the full pass agrees with its NLL.
"""
import numpy as np
import pytest

from ctpwa_b200 import workloads
from oracle.binding import Oracle

pytestmark = pytest.mark.gpu

CASES = {"pipi_rho": (30_000, 5_000, 0), "pipi_3rho": (40_000, 5_000, 1_000), "kkpi": (40_000, 5_000, 1_000)}


def _setup(tmp_path, name, sizes=None, seed=5):
    import torch
    import ctpwa_b200

    nph, nda, nbk = sizes or CASES[name]
    cfg = workloads.make(name, tmp_path, n_phsp=nph, n_data=nda, n_bkg=nbk, accept_reject=False, seed=seed)
    ana = ctpwa_b200.analysis(cfg)
    nV = ana.getNVector()
    p = workloads.true_params(nV, ana.getFreeResParams()[0].numpy())
    p[2 * nV:] *= 1 + 0.01 * np.random.default_rng(seed).standard_normal(p.size - 2 * nV)
    return cfg, ana, p, torch.tensor(p, dtype=torch.float64, device="cuda")


def _other_couplings(p, nV, seed):
    q = p.copy()
    rng = np.random.default_rng(seed)
    q[1:nV] *= 1 + 0.2 * rng.standard_normal(nV - 1)
    q[nV + 1:2 * nV] += 0.3 * rng.standard_normal(nV - 1)
    return q


def _close(n1, g1, n0, g0, rel=1e-10, grel=1e-9):
    n1, n0 = float(n1), float(n0)
    g1 = g1.cpu().numpy() if hasattr(g1, "cpu") else np.asarray(g1)
    g0 = g0.cpu().numpy() if hasattr(g0, "cpu") else np.asarray(g0)
    assert abs(n1 - n0) <= rel * max(1.0, abs(n0)), (n1, n0)
    assert np.max(np.abs(g1 - g0)) <= grel * np.max(np.abs(g0)), np.max(np.abs(g1 - g0)) / np.max(np.abs(g0))


@pytest.mark.parametrize("name", list(CASES))
def test_cached_matches_full_pass_and_oracle(tmp_path, name):
    import torch

    cfg, ana, p, pt = _setup(tmp_path, name)
    nV = ana.getNVector()
    assert not ana.hasNormalisationCache()
    ms = ana.cacheNormalisation(pt)
    assert ana.hasNormalisationCache() and ms > 0
    orc = Oracle(cfg)
    for q in (p, _other_couplings(p, nV, 1), _other_couplings(p, nV, 2)):
        qt = torch.tensor(q, dtype=torch.float64, device="cuda")
        n0, g0 = ana.getNLLAndGrad(qt, "fp64")
        n1, g1 = ana.getNLLAndGrad(qt, "fp64", cached=True)
        _close(n1, g1, n0, g0)
        onll, og, _ = orc.nll_grad(q)
        _close(n1, g1, onll, og)
        nm, gm = ana.getNLLAndGrad(qt, "mixed", cached=True)
        assert abs(float(nm) - onll) < 1e-3, (float(nm), onll)
        assert np.max(np.abs(gm.cpu().numpy() - og)) <= 1e-4 * np.max(np.abs(og))


def test_weighted_phase_space(tmp_path):
    import torch
    import ctpwa_b200
    from test_gpu_parity import _weighted_config

    cfg = _weighted_config(tmp_path, 20_011, 3_001, 507, seed=43, short_bkg=False)
    ana = ctpwa_b200.analysis(cfg)
    orc = Oracle(cfg)
    nV = ana.getNVector()
    p = workloads.true_params(nV, ana.getFreeResParams()[0].numpy())
    ana.cacheNormalisation(torch.tensor(p, dtype=torch.float64, device="cuda"))
    for q in (p, _other_couplings(p, nV, 3)):
        qt = torch.tensor(q, dtype=torch.float64, device="cuda")
        n1, g1 = ana.getNLLAndGrad(qt, "fp64", cached=True)
        onll, og, _ = orc.nll_grad(q)
        _close(n1, g1, onll, og)
        n0, g0 = ana.getNLLAndGrad(qt, "fp64")
        _close(n1, g1, n0, g0)


def test_other_resonance_parameters(tmp_path):
    import torch

    cfg, ana, p, pt = _setup(tmp_path, "kkpi")
    nV = ana.getNVector()
    ana.cacheNormalisation(pt)
    q = p.copy()
    q[2 * nV] *= 1 + 1e-12
    qt = torch.tensor(q, dtype=torch.float64, device="cuda")
    # cached entry point: flagged invalid, not silently wrong
    n, g = ana.getNLLAndGrad(qt, "fp64", cached=True)
    assert float(n) == 1e30 and not bool(g.abs().max() > 0)
    # host entry point: the full pass for these parameters, the cache for the cached ones
    nh, gh = ana.getNLLHost(q, "fp64")
    n0, g0 = ana.getNLLAndGrad(qt, "fp64")
    assert nh == float(n0) and np.array_equal(gh, g0.cpu().numpy())
    nh2, gh2 = ana.getNLLHost(p, "fp64")
    nc, gc = ana.getNLLAndGrad(pt, "fp64", cached=True)
    assert nh2 == float(nc) and np.array_equal(gh2, gc.cpu().numpy())
    # the cache did not change the full pass
    ana.clearNormalisationCache()
    assert not ana.hasNormalisationCache()
    with pytest.raises(RuntimeError):
        ana.getNLLAndGrad(pt, "fp64", cached=True)
    n2, g2 = ana.getNLLAndGrad(pt, "fp64")
    _close(n2, g2, nc, gc)


def test_fit_with_fixed_resonance_parameters(tmp_path):
    import torch

    cfg, ana, p, pt = _setup(tmp_path, "pipi_3rho", sizes=(60_000, 8_000, 0))
    nV, n = ana.getNVector(), ana.getNParams()
    free = np.zeros(n, dtype=np.uint8)
    free[1:nV] = 1
    free[nV + 1:2 * nV] = 1
    x0 = _other_couplings(p, nV, 4)
    assert not ana.hasNormalisationCache()
    x, nll, ne, _, status, _ = ana.fit(x0, free=free, max_evals=300, precision="fp64")
    assert ana.hasNormalisationCache()
    assert status in (0, 1), status
    assert np.array_equal(x[2 * nV:], x0[2 * nV:])
    # the full pass agrees with the fit's NLL at its end point and sees a minimum in the couplings
    ana.clearNormalisationCache()
    n0, g0 = ana.getNLLAndGrad(torch.tensor(x, dtype=torch.float64, device="cuda"), "fp64")
    assert abs(float(n0) - nll) <= 1e-10 * abs(nll)
    assert np.max(np.abs(g0.cpu().numpy()[free.astype(bool)])) < 1e-2


def test_model_without_free_resonance_parameters(tmp_path):
    """Every resonance parameter fixed in the configuration (no theta at
    all): the cache holds for every evaluation, including the fit's."""
    import torch
    import ctpwa_b200

    cfg = workloads.make("pipi_3rho", tmp_path, n_phsp=30_000, n_data=4_000, n_bkg=500, accept_reject=False, seed=9)
    text = open(cfg).read()
    assert ", free: [0, 1]" in text
    open(cfg, "w").write(text.replace(", free: [0, 1]", ""))
    ana = ctpwa_b200.analysis(cfg)
    assert ana.getNFreeTheta() == 0
    nV = ana.getNVector()
    p = workloads.true_params(nV, [])
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    ana.cacheNormalisation(pt)
    orc = Oracle(cfg)
    for q in (p, _other_couplings(p, nV, 5)):
        qt = torch.tensor(q, dtype=torch.float64, device="cuda")
        n1, g1 = ana.getNLLAndGrad(qt, "fp64", cached=True)
        _close(n1, g1, *ana.getNLLAndGrad(qt, "fp64"))
        onll, og, _ = orc.nll_grad(q)
        _close(n1, g1, onll, og)
    ana.clearNormalisationCache()
    x, nll, *_ = ana.fit(_other_couplings(p, nV, 6), max_evals=300, precision="fp64")
    assert ana.hasNormalisationCache()
    n0, _ = ana.getNLLAndGrad(torch.tensor(x, dtype=torch.float64, device="cuda"), "fp64")
    assert abs(float(n0) - nll) <= 1e-10 * abs(nll)
