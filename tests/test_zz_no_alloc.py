"""Allocation-free evaluation entry point (ctpwa_nll_grad_static).

Some callers cannot let a library allocate device memory for them, for
example a host program that has handed all device memory to its own pool
allocator, or a serving loop that counts every device byte against a fixed
budget. ctpwa_nll_grad_static evaluates the NLL and gradient with its scratch
in a fixed array compiled into the library instead of per-handle buffers.
These tests call it through the C ABI and check it against ctpwa_nll_grad
(the regular entry point) on two calls in a row, for both precisions. Both
entry points launch the same kernels with the same grid and the same fixed
reduction order, so the results must be bit-identical. This file is
collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest

from ctpwa_b200 import workloads

pytestmark = pytest.mark.gpu

CASES = {"pipi_rho": (20_000, 5_000, 0), "kkpi": (200_000, 20_000, 2_000)}


def _static_call(ana, pt, prec, nll=None, grad=None):
    import torch

    if nll is None:
        nll = torch.empty((), dtype=torch.float64, device=pt.device)
        grad = torch.empty_like(pt)
    stream = torch.cuda.current_stream(pt.device).cuda_stream
    rc = ana._lib.ctpwa_nll_grad_static(ana._h, pt.data_ptr(), nll.data_ptr(), grad.data_ptr(), prec,
                                        ctypes.c_void_p(stream))
    return rc, nll, grad


@pytest.mark.parametrize("name", list(CASES))
def test_static_scratch_matches_regular_entry(tmp_path, name):
    import torch
    import ctpwa_b200

    nph, nda, nbk = CASES[name]
    cfg = workloads.make(name, tmp_path, n_phsp=nph, n_data=nda, n_bkg=nbk, accept_reject=False, seed=7)
    ana = ctpwa_b200.analysis(cfg)
    nV = ana.getNVector()
    p0 = workloads.true_params(nV, ana.getFreeResParams()[0].numpy())
    rng = np.random.default_rng(21)
    for prec in (0, 1):
        # two calls in a row at different parameters: the second must not see the first's scratch
        for call in range(2):
            p = p0.copy()
            p[2 * nV:] *= 1 + 0.01 * rng.standard_normal(p.size - 2 * nV)
            p[:2 * nV] *= 1 + 0.05 * call
            pt = torch.tensor(p, dtype=torch.float64, device="cuda")
            rc, n_s, g_s = _static_call(ana, pt, prec)
            assert rc == 0, ana._lib.ctpwa_last_error(ana._h)
            n_r, g_r = ana.getNLLAndGrad(pt, prec)
            torch.cuda.synchronize()
            assert float(n_s) == float(n_r), (prec, call, float(n_s), float(n_r))
            assert torch.equal(g_s, g_r), (prec, call, float((g_s - g_r).abs().max()))


def test_static_scratch_allocates_nothing(tmp_path):
    """After the first call (which looks the array's address up), further
    calls change neither the device's free memory nor torch's pool."""
    import torch
    import ctpwa_b200

    cfg = workloads.make("kkpi", tmp_path, n_phsp=50_000, n_data=5_000, n_bkg=500, accept_reject=False, seed=9)
    ana = ctpwa_b200.analysis(cfg)
    p = workloads.true_params(ana.getNVector(), ana.getFreeResParams()[0].numpy())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    nll = torch.empty((), dtype=torch.float64, device="cuda")
    grad = torch.empty_like(pt)
    for prec in (0, 1):
        assert _static_call(ana, pt, prec, nll, grad)[0] == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    for i in range(20):
        assert _static_call(ana, pt, i % 2, nll, grad)[0] == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_reserved() == reserved0


def _many_rho_config(tmp_path, nres):
    """Three pi pi chains with `nres` BWR states each (3 nres amplitude
    columns): a model whose per-CTA partial rows are long."""
    cfg = workloads.make("pipi_3rho", tmp_path, n_phsp=100_000, n_data=5_000, n_bkg=0, accept_reject=False, seed=10)
    text = open(cfg).read()
    names = [f"r{i}" for i in range(nres)]
    text = text.replace("[rho770, rho1450, rho1700]", "[" + ", ".join(names) + "]")
    head = text[:text.index("Resonances:")]
    res = "Resonances:\n" + "".join(
        f"  {n}: {{J: 1, P: -1, model: BWR, parameters: [{0.7 + 0.09 * i:.3f}, {0.12 + 0.01 * i:.3f}], free: [0, 1]}}\n"
        for i, n in enumerate(names))
    open(cfg, "w").write(head + res)
    return cfg


def test_static_scratch_rejects_models_that_do_not_fit(tmp_path, monkeypatch):
    """A model whose partial rows exceed the fixed array is rejected with
    CTPWA_ERR_ARG and a message pointing to the regular entry point, while a
    launch shape that fits still evaluates bit-identically."""
    import torch
    import ctpwa_b200

    # 32-thread CTAs, at least 16 per SM (one partial row each): >= 2368 rows
    # on 148 SMs, x (2 + 2 x 51 + 34) sums > the 2 MiB array
    monkeypatch.setenv("CTPWA_MX_BLOCK", "32")
    monkeypatch.setenv("CTPWA_MX_MINB", "16")
    ana = ctpwa_b200.analysis(_many_rho_config(tmp_path, 17))
    assert ana.isValid()
    nacc = 2 + 2 * ana.getNVector() + ana.getNFreeTheta()
    p = workloads.true_params(ana.getNVector(), ana.getFreeResParams()[0].numpy())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    rc, _, _ = _static_call(ana, pt, 1)
    assert rc == -3, (rc, nacc)
    msg = ana._lib.ctpwa_last_error(ana._h)
    assert b"use ctpwa_nll_grad" in msg and b"bytes of scratch" in msg
    # the plain path's grid (2 CTAs per SM) fits
    rc, n_s, g_s = _static_call(ana, pt, 0)
    assert rc == 0, ana._lib.ctpwa_last_error(ana._h)
    n_r, g_r = ana.getNLLAndGrad(pt, 0)
    torch.cuda.synchronize()
    assert float(n_s) == float(n_r) and torch.equal(g_s, g_r)


def test_static_scratch_rejects_bad_arguments(tmp_path):
    import torch
    import ctpwa_b200

    cfg = workloads.make("pipi_rho", tmp_path, n_phsp=4_000, n_data=1_000, n_bkg=0, accept_reject=False, seed=8)
    ana = ctpwa_b200.analysis(cfg)
    pt = torch.zeros(ana.getNParams(), dtype=torch.float64, device="cuda")
    out = torch.empty(1 + ana.getNParams(), dtype=torch.float64, device="cuda")
    rc = ana._lib.ctpwa_nll_grad_static(ana._h, pt.data_ptr(), out.data_ptr(), out[1:].data_ptr(), 7, None)
    assert rc == -3
    assert b"precision" in ana._lib.ctpwa_last_error(ana._h)
    rc = ana._lib.ctpwa_nll_grad_static(ana._h, None, out.data_ptr(), out[1:].data_ptr(), 0, None)
    assert rc == -3
