"""Generated angular kernels against the interpreted one.

The angular tables (spin-orbit vertex tensors contracted along each chain)
and the kinematic cache are built at handle creation either by the kernels
generated per model (one straight-line kernel per angular group, tensor
shapes fixed at compile time; the default) or by the interpreter
`ag_group_kernel` (`CTPWA_ANGULAR_INTERP=1`). Both evaluate the same
formulas in the same order; the test requires the per-event FP64
intensities of every sample to agree to 1e-13 relative at random couplings
(every angular plane contributes) and the FP64 / mixed NLL and gradient to
agree to 1e-12 relative, on every bundled model (identical particles in
ksks), the feature config and a J/psi polarisation mask; and both decide the
polarisation pairing of the fused kernels alike.
"""
import numpy as np
import pytest

from ctpwa_b200 import workloads

pytestmark = pytest.mark.gpu

MODELS = {"pipi_rho": (30_000, 5_000, 0), "pipi_3rho": (30_000, 5_000, 2_000), "kkpi": (30_011, 5_003, 1_001),
          "ksks": (20_000, 4_000, 0)}


def _pol_mask(text):
    return text.replace("Jpsi: {J: 1, P: -1, mass: 3.0969}", "Jpsi: {J: 1, P: -1, mass: 3.0969, polarization: [1, -1]}")


def _compare(cfg, monkeypatch, seeds=(1, 2)):
    import torch
    import ctpwa_b200

    monkeypatch.delenv("CTPWA_ANGULAR_INTERP", raising=False)
    gen = ctpwa_b200.analysis(cfg)
    monkeypatch.setenv("CTPWA_ANGULAR_INTERP", "1")
    itp = ctpwa_b200.analysis(cfg)
    monkeypatch.delenv("CTPWA_ANGULAR_INTERP")
    assert gen.isValid() and itp.isValid()
    # the polarisation-pairing decision: from the maxima the generated
    # kernels gather while writing, and from the separate check kernel
    assert gen.launchShape() == itp.launchShape()
    nV = gen.getNVector()
    base = workloads.true_params(nV, gen.getFreeResParams()[0].numpy())
    for seed in seeds:
        rng = np.random.default_rng(seed)
        p = base.copy()
        p[1:2 * nV] = rng.uniform(-1, 1, 2 * nV - 1)
        p[nV] = 0.0
        pt = torch.tensor(p, dtype=torch.float64, device="cuda")
        for kind, n in enumerate(gen.getNEvents()):
            if n == 0:
                continue
            a = gen.getIntensity(pt, kind).cpu().numpy()
            b = itp.getIntensity(pt, kind).cpu().numpy()
            assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(b)), (cfg, kind, np.max(np.abs(a - b)))
        for prec in ("fp64", "mixed"):
            na, ga = gen.getNLLAndGrad(pt, prec)
            nb, gb = itp.getNLLAndGrad(pt, prec)
            assert abs(float(na) - float(nb)) <= 1e-12 * abs(float(nb)), (cfg, prec, float(na), float(nb))
            assert float((ga - gb).abs().max()) <= 1e-12 * float(gb.abs().max()) + 1e-300, (cfg, prec)


@pytest.mark.parametrize("name", list(MODELS))
def test_generated_angular_tables_match_interpreter(tmp_path, monkeypatch, name):
    nph, nda, nbk = MODELS[name]
    cfg = workloads.make(name, tmp_path, n_phsp=nph, n_data=nda, n_bkg=nbk, accept_reject=False, seed=5)
    _compare(cfg, monkeypatch)


def test_generated_angular_tables_with_polarisation_mask(tmp_path, monkeypatch):
    cfg = workloads.make("kkpi", tmp_path, n_phsp=20_000, n_data=3_000, n_bkg=0, accept_reject=False, seed=6)
    with open(cfg) as f:
        text = _pol_mask(f.read())
    with open(cfg, "w") as f:
        f.write(text)
    _compare(cfg, monkeypatch, seeds=(3,))


def test_generated_angular_tables_feature_config(tmp_path, monkeypatch):
    from test_gpu_parity import _features_config

    monkeypatch.chdir(tmp_path)
    _compare(_features_config(tmp_path), monkeypatch, seeds=(4,))
