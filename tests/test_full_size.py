"""The benchmark workloads at their full sizes against the FP64 oracle.

J/psi -> K+ K- pi0 with 10M phase-space, 1M data (accept-reject against the
model) and 100k background events (weight 0.3), generated on the GPU; the
oracle reads the same events. FP64 path: NLL 1e-10 relative, gradient 1e-9
of its largest component. Mixed form: |dNLL| < 1e-3 against the FP64 oracle
(not against the device FP64 path) and gradient 1e-4 of its largest
component.
"""
import numpy as np
import pytest

from ctpwa_b200 import toymc, workloads
from oracle.binding import Oracle

pytestmark = pytest.mark.gpu


def test_full_kkpi_workload_against_oracle(tmp_path):
    import torch
    import ctpwa_b200

    n_p, n_d, n_b, w_b = workloads.SIZES["kkpi"]
    cfg, phsp, data, bkg, wts = workloads.make_device_samples("kkpi", tmp_path / "dev", n_p, n_d, n_bkg=n_b,
                                                              bkg_weight=w_b, seed=3)
    ana = ctpwa_b200.analysis.from_device(cfg, phsp, data, bkg, weights=wts)
    d = tmp_path / "host"
    d.mkdir()
    for name, t in (("phsp", phsp), ("data", data), ("bkg", bkg)):
        toymc.write_npy(d / f"{name}.npy", t.cpu().numpy())
    del phsp, data, bkg, wts
    hcfg = d / "config.yml"
    hcfg.write_text(workloads.config_text("kkpi", str(d / "phsp.npy"), str(d / "data.npy"), str(d / "bkg.npy"), w_b))
    orc = Oracle(str(hcfg))
    assert orc.nev == tuple(int(x) for x in ana.getNEvents())
    nV = ana.getNVector()
    p = workloads.true_params(nV, ana.getFreeResParams()[0].numpy())
    p[2 * nV:] *= 1 + 0.005 * np.random.default_rng(8).standard_normal(p.size - 2 * nV)
    onll, og, _ = orc.nll_grad(p)
    orc.close()
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    nll, g = ana.getNLLAndGrad(pt, "fp64")
    assert abs(float(nll) - onll) <= 1e-10 * abs(onll), (float(nll), onll)
    assert np.max(np.abs(g.cpu().numpy() - og)) <= 1e-9 * np.max(np.abs(og))
    nmx, gmx = ana.getNLLAndGrad(pt, "mixed")
    assert abs(float(nmx) - onll) < 1e-3, (float(nmx), onll)
    assert np.max(np.abs(gmx.cpu().numpy() - og)) <= 1e-4 * np.max(np.abs(og))


def _device_and_oracle(tmp_path, name, n_p, n_d, n_b, w_b, seed):
    """The workload generated on the GPU (data by accept-reject against the
    model plus the subtracted background) as a device handle, and the oracle
    on the same events written to .npy files."""
    import ctpwa_b200

    cfg, phsp, data, bkg, wts = workloads.make_device_samples(name, tmp_path / "dev", n_p, n_d, n_bkg=n_b,
                                                              bkg_weight=w_b, seed=seed)
    ana = ctpwa_b200.analysis.from_device(cfg, phsp, data, bkg, weights=wts)
    d = tmp_path / "host"
    d.mkdir()
    samples = [("phsp", phsp), ("data", data)] + ([("bkg", bkg)] if bkg is not None else [])
    for label, t in samples:
        toymc.write_npy(d / f"{label}.npy", t.cpu().numpy())
    del phsp, data, bkg, wts
    hcfg = d / "config.yml"
    hcfg.write_text(workloads.config_text(name, str(d / "phsp.npy"), str(d / "data.npy"),
                                          str(d / "bkg.npy") if n_b else None, w_b if n_b else None))
    orc = Oracle(str(hcfg))
    assert orc.nev == tuple(int(x) for x in ana.getNEvents())
    return ana, orc


def test_single_rho_workload_at_its_sizes(tmp_path):
    """J/psi -> pi+ pi- pi0 with rho(770), 200k phase space / 20k data: FP64
    NLL and gradient against the oracle (1e-10 / 1e-9), the mixed form
    (|dNLL| < 1e-3 against the oracle), and the exact Hessian against the
    oracle's Richardson-extrapolated differences (1e-8 of the largest entry)."""
    import torch

    ana, orc = _device_and_oracle(tmp_path, "pipi_rho", 200_000, 20_000, 0, None, seed=7)
    nV = ana.getNVector()
    p = workloads.true_params(nV, ana.getFreeResParams()[0].numpy())
    p[2 * nV:] *= 1 + 0.01 * np.random.default_rng(3).standard_normal(p.size - 2 * nV)
    onll, og, _ = orc.nll_grad(p)
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    nll, g = ana.getNLLAndGrad(pt, "fp64")
    assert abs(float(nll) - onll) <= 1e-10 * abs(onll), (float(nll), onll)
    assert np.max(np.abs(g.cpu().numpy() - og)) <= 1e-9 * np.max(np.abs(og))
    nmx, _ = ana.getNLLAndGrad(pt, "mixed")
    assert abs(float(nmx) - onll) < 1e-3, (float(nmx), onll)
    H = ana.getHessian(pt).cpu().numpy()
    Ho = orc.hessian_fd(p)
    assert np.max(np.abs(H - Ho)) <= 1e-8 * np.max(np.abs(Ho))
    orc.close()


def test_three_chain_rho_workload_at_its_sizes(tmp_path):
    """J/psi -> pi+ pi- pi0 with three rho chains x three rho states, 5M phase
    space / 500k data / 50k background at weight 0.8: FP64 NLL and gradient
    against the oracle (1e-10 / 1e-9) and the mixed form (|dNLL| < 1e-3
    against the oracle). Its Hessian is compared with the reference's own
    CUDA build (test_reference_cuda.py)."""
    import torch

    ana, orc = _device_and_oracle(tmp_path, "pipi_3rho", 5_000_000, 500_000, 50_000, 0.8, seed=9)
    nV = ana.getNVector()
    p = workloads.true_params(nV, ana.getFreeResParams()[0].numpy())
    p[2 * nV:] *= 1 + 0.005 * np.random.default_rng(4).standard_normal(p.size - 2 * nV)
    onll, og, _ = orc.nll_grad(p)
    orc.close()
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    nll, g = ana.getNLLAndGrad(pt, "fp64")
    assert abs(float(nll) - onll) <= 1e-10 * abs(onll), (float(nll), onll)
    assert np.max(np.abs(g.cpu().numpy() - og)) <= 1e-9 * np.max(np.abs(og))
    nmx, gmx = ana.getNLLAndGrad(pt, "mixed")
    assert abs(float(nmx) - onll) < 1e-3, (float(nmx), onll)
    assert np.max(np.abs(gmx.cpu().numpy() - og)) <= 1e-4 * np.max(np.abs(og))
