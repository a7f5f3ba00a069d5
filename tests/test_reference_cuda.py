"""The device path against the reference's own CUDA build on identical inputs.

The reference extension is built from its unmodified sources by
oracle/refcuda/build.py (FP64 build, complex<double>) and driven through its
public API (ctpwa.analysis, getNLL + autograd, getHessian, the layout
queries) in a child process. Both sides read the same `.dat` sample files and
the same config.

Tolerances: parameter layout (names, counts, default ranges) identical; FP64
NLL 1e-10 relative and gradient 1e-9 of its largest component; the Hessian
1e-7 of its largest entry (the reference forms it from Gram products and
second lineshape derivatives, this library by forward mode over the adjoint
pass); the mixed form |dNLL| < 1e-3 against the reference FP64 build.
"""
import numpy as np
import pytest

from ctpwa_b200 import workloads
from oracle import refcuda

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refcuda.available("f64"), reason="reference CUDA build not present")]

# workload: (phase space, data, background) events; pipi_rho at its benchmark sizes
CASES = {"pipi_rho": (200_000, 20_000, 0), "pipi_3rho": (500_000, 50_000, 5_000),
         "kkpi": (1_000_000, 100_000, 10_000)}


def _points(ana, nseed=2):
    nV = ana.getNVector()
    p0 = workloads.true_params(nV, ana.getFreeResParams()[0].numpy())
    pts = [p0]
    rng = np.random.default_rng(17)
    for _ in range(nseed - 1):
        p = p0.copy()
        p[2 * nV:] *= 1 + 0.02 * rng.standard_normal(p.size - 2 * nV)
        p[2:2 * nV] *= 1 + 0.1 * rng.standard_normal(2 * nV - 2)
        pts.append(p)
    return pts


@pytest.fixture(scope="module", params=list(CASES))
def case(request, tmp_path_factory):
    import ctpwa_b200

    name = request.param
    nph, nda, nbk = CASES[name]
    d = tmp_path_factory.mktemp("ref_" + name)
    cfg = workloads.make(name, d, n_phsp=nph, n_data=nda, n_bkg=nbk, accept_reject=True, seed=31)
    dcfg = refcuda.dat_config(cfg)
    ana = ctpwa_b200.analysis(dcfg)
    assert ana.isValid()
    pts = _points(ana)
    ref = refcuda.run("f64", dcfg, pts, hessian=True)
    return name, ana, pts, ref


def test_layout_matches_reference_build(case):
    name, ana, _, ref = case
    assert ana.getNVector() == ref["nV"]
    assert ana.getNFreeTheta() == ref["nT"]
    assert list(ana.getParamNames()) == list(ref["names"]), name
    np.testing.assert_array_equal(ana.getFreeResParams().numpy(), ref["free_res_params"])


def test_fp64_nll_grad_match_reference_build(case):
    import torch

    name, ana, pts, ref = case
    for i, p in enumerate(pts):
        pt = torch.tensor(p, dtype=torch.float64, device="cuda")
        nll, g = ana.getNLLAndGrad(pt, "fp64")
        rn, rg = float(ref["nll"][i]), ref["grad"][i]
        assert abs(float(nll) - rn) <= 1e-10 * max(1.0, abs(rn)), (name, i, float(nll), rn)
        g = g.cpu().numpy()
        assert np.max(np.abs(g - rg)) <= 1e-9 * np.max(np.abs(rg)), (name, i, np.max(np.abs(g - rg)) / np.max(np.abs(rg)))


def test_mixed_nll_within_budget_of_reference_build(case):
    import torch

    name, ana, pts, ref = case
    for i, p in enumerate(pts):
        pt = torch.tensor(p, dtype=torch.float64, device="cuda")
        nll, g = ana.getNLLAndGrad(pt, "mixed")
        assert abs(float(nll) - float(ref["nll"][i])) < 1e-3, (name, i)
        rg = ref["grad"][i]
        assert np.max(np.abs(g.cpu().numpy() - rg)) <= 1e-4 * np.max(np.abs(rg))


def test_hessian_matches_reference_build(case):
    import torch

    name, ana, pts, ref = case
    for i, p in enumerate(pts):
        H = ana.getHessian(torch.tensor(p, dtype=torch.float64, device="cuda")).cpu().numpy()
        R = ref["hessian"][i]
        scale = np.max(np.abs(R))
        assert np.max(np.abs(H - R)) <= 1e-7 * scale, (name, i, np.max(np.abs(H - R)) / scale)
