"""The device path against the reference's own CUDA build on identical inputs.

The reference extension is built from its unmodified sources by
oracle/refcuda/build.py (FP64 build, complex<double>) and driven through its
public API (ctpwa.analysis, getNLL + autograd, getHessian, the layout
queries) in a child process. Both sides read the same `.dat` sample files and
the same config.

The reference's FP64 build rounds one quantity to single precision: the
scale (W_data - W_bkg) / pf of the phase-space term of the coupling gradient
(both operands cast to float and divided in float, src/Analysis.cu:1159-1162).
That moves its coupling gradients by ~6e-8 of the phase-space term, which
after the data / phase-space cancellation is up to ~1e-6 of the gradient, and
puts the same rounding noise into finite differences of its gradient. This
library keeps the scale in FP64. The comparison therefore applies the
reference's rounding to this library's FP64 shard sums (`_reference_rounded`)
and checks that against the reference to 1e-9; the unrounded FP64 gradient is
checked against it within the size of the rounding.

Tolerances: parameter layout (names, counts, default ranges) identical; FP64
NLL 1e-10 relative; gradient with the reference's rounding 1e-9 of its
largest component; the exact Hessian 2e-5 of its largest entry against
central differences of the reference's gradient with its rounding taken out
(the differences' own truncation and rounding error); the mixed form
|dNLL| < 1e-3 against the reference FP64 build.
"""
import numpy as np
import pytest

from ctpwa_b200 import workloads
from oracle import refcuda

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refcuda.available("f64"), reason="reference CUDA build not present")]



def _veq_pol(text):
    """Schema features beyond the benchmark models: a polarisation mask on the
    J/psi (m = +-1 only, src/Analysis.cu:4249-4322) and a var_equal group
    (two resonance widths share one fitted parameter, src/AmpGen.cu:2244-2342)."""
    text = text.replace("Jpsi: {J: 1, P: -1, mass: 3.0969}", "Jpsi: {J: 1, P: -1, mass: 3.0969, polarization: [1, -1]}")
    return text.replace("Resonances:", "Constraints:\n  var_equal:\n    - [Kst892_width, Kst1410_width]\nResonances:", 1)


# case: (workload, (phase space, data, background) events, config transform);
# pipi_rho at its benchmark sizes (config 1), the others on samples of theirs
CASES = {"pipi_rho": ("pipi_rho", (200_000, 20_000, 0), None),
         "pipi_3rho": ("pipi_3rho", (500_000, 50_000, 5_000), None),
         "kkpi": ("kkpi", (1_000_000, 100_000, 10_000), None),
         "kkpi_veq_pol": ("kkpi", (200_000, 20_000, 2_000), _veq_pol)}


def _reference_rounded(ana, p):
    """(nll, grad) of this library in FP64 with the phase-space gradient scale
    s = (W_data - W_bkg) / pf rounded as the reference's FP64 build rounds it:
    float(W_data - W_bkg) / float(pf) in single precision
    (src/Analysis.cu:1159-1162). Applied by scaling the phase-space coupling
    sums of this library's shard sums by s_f / s before the finalisation."""
    import torch

    pt = torch.as_tensor(p, dtype=torch.float64).cuda()
    S = ana.getShardSums(pt, "fp64").cpu().numpy().copy()
    nacc = (S.size - 4) // 3
    nA = len(ana.getAmplitudeNames())
    n_phsp, w_data, w_bkg = S[3 * nacc], S[3 * nacc + 2], S[3 * nacc + 3]
    pf = S[1] / n_phsp
    if not (pf > 1e-30 and np.isfinite(pf)):
        pf = 1e-30
    weff = w_data - w_bkg
    s_f = float(np.float32(weff) / np.float32(pf))
    S[2:2 + 2 * nA] *= s_f / (weff / pf)
    nll, g = ana.finalizeShardSums(pt, torch.from_numpy(S).cuda())
    return float(nll), g.cpu().numpy()


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
    import torch
    import ctpwa_b200

    name = request.param
    wl, (nph, nda, nbk), transform = CASES[name]
    d = tmp_path_factory.mktemp("ref_" + name)
    cfg = workloads.make(wl, d, n_phsp=nph, n_data=nda, n_bkg=nbk, accept_reject=True, seed=31)
    if transform:
        with open(cfg) as f:
            text = transform(f.read())
        with open(cfg, "w") as f:
            f.write(text)
    dcfg = refcuda.dat_config(cfg)
    ana = ctpwa_b200.analysis(dcfg)
    assert ana.isValid()
    pts = _points(ana)
    # central differences of the reference build's own gradient at the first point
    p0 = pts[0]
    steps = [2.5e-6 * max(abs(x), 1e-2) for x in p0]
    fd = []
    for i, h in enumerate(steps):
        for sgn in (1.0, -1.0):
            q = p0.copy()
            q[i] += sgn * h
            fd.append(q)
    ref = refcuda.run("f64", dcfg, pts + fd, hessian=True)
    # the reference's single-precision scale taken out of its gradient at each
    # difference point: g_ref - (g_rounded - g_fp64) of this library there
    G = []
    for q, gq in zip(fd, ref["grad"][len(pts):]):
        _, g_r = _reference_rounded(ana, q)
        _, g_e = ana.getNLLAndGrad(torch.tensor(q, dtype=torch.float64, device="cuda"), "fp64")
        G.append(gq - (g_r - g_e.cpu().numpy()))
    H = np.array([(G[2 * i] - G[2 * i + 1]) / (2 * steps[i]) for i in range(len(p0))])
    ref["hessian_fd"] = 0.5 * (H + H.T)
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
        scale = np.max(np.abs(rg))
        # with the reference's single-precision phase-space scale applied
        n_r, g_r = _reference_rounded(ana, p)
        assert abs(n_r - float(nll)) == 0.0
        assert np.max(np.abs(g_r - rg)) <= 1e-9 * scale, (name, i, np.max(np.abs(g_r - rg)) / scale)
        # the FP64 gradient: the theta components directly, the coupling
        # components within the size of that rounding
        n2 = 2 * ana.getNVector()
        assert np.max(np.abs(g[n2:] - rg[n2:])) <= 1e-9 * scale, (name, i)
        assert np.max(np.abs(g - rg)) <= 2.0 * np.max(np.abs(g_r - g)) + 1e-9 * scale, (name, i)


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
    """The exact Hessian against central differences of the reference build's
    own gradient (its single-precision phase-space scale taken out, see the
    module docstring), over the parameters a fit moves (the first coupling is held
    fixed; differences along it are not meaningful for the reference). The
    reference's analytic getHessian is recorded beside it: it deviates from
    the differences of its own gradient by up to ~5e-4 of the largest entry
    (mass-mass entries of the resonance parameters)."""
    import torch

    name, ana, pts, ref = case
    H = ana.getHessian(torch.tensor(pts[0], dtype=torch.float64, device="cuda")).cpu().numpy()
    n = ana.getNVector()
    free = [j for j in range(H.shape[0]) if j not in (0, n)]
    F = ref["hessian_fd"][np.ix_(free, free)]
    Hf = H[np.ix_(free, free)]
    scale = np.max(np.abs(F))
    assert np.max(np.abs(Hf - F)) <= 2e-5 * scale, (name, np.max(np.abs(Hf - F)) / scale)
    R = ref["hessian"][0][np.ix_(free, free)]
    assert np.max(np.abs(R - F)) <= 5e-3 * scale  # the reference's own analytic Hessian, for the record
