"""Allocation-free evaluation entry point (ctpwa_nll_grad_static).

Some callers cannot let a library allocate device memory for them, for
example a host program that has handed all device memory to its own pool
allocator, or a serving loop that counts every device byte against a fixed
budget. ctpwa_nll_grad_static evaluates the NLL and gradient with its scratch
in a fixed array compiled into the library instead of per-handle buffers.
These tests call it through the C ABI and check it against ctpwa_nll_grad
(the regular entry point) on two calls in a row, for both precisions, with
the tolerances of the other GPU tests. This file is collected last so that a
run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from ctpwa_b200 import workloads

pytestmark = pytest.mark.gpu

CASES = {"pipi_rho": (20_000, 5_000, 0), "kkpi": (200_000, 20_000, 2_000)}


def _static_call(ana, pt, prec):
    import torch

    nll = torch.empty((), dtype=torch.float64, device=pt.device)
    grad = torch.empty_like(pt)
    stream = torch.cuda.current_stream(pt.device).cuda_stream
    rc = ana._lib.ctpwa_nll_grad_static(ana._h, pt.data_ptr(), nll.data_ptr(), grad.data_ptr(), prec,
                                        ctypes.c_void_p(stream))
    assert rc == 0, ana._lib.ctpwa_last_error(ana._h)
    return nll, grad


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
    for prec, rtol_nll, rtol_g, atol_nll in ((0, 1e-10, 1e-9, 0.0), (1, 0.0, 1e-4, 1e-3)):
        # two calls in a row at different parameters: the second must not see the first's scratch
        for call in range(2):
            p = p0.copy()
            p[2 * nV:] *= 1 + 0.01 * rng.standard_normal(p.size - 2 * nV)
            p[:2 * nV] *= 1 + 0.05 * call
            pt = torch.tensor(p, dtype=torch.float64, device="cuda")
            n_s, g_s = _static_call(ana, pt, prec)
            n_r, g_r = ana.getNLLAndGrad(pt, prec)
            torch.cuda.synchronize()
            n_s, n_r = float(n_s), float(n_r)
            assert abs(n_s - n_r) <= max(atol_nll, rtol_nll * max(1.0, abs(n_r))), (prec, call, n_s, n_r)
            scale = float(g_r.abs().max())
            assert float((g_s - g_r).abs().max()) <= rtol_g * scale, (prec, call)


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
