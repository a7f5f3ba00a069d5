"""Device path vs the FP64 CPU oracle on the same seeded inputs.

Tolerances: plain FP64 path 1e-10 relative on the NLL and 1e-9 (relative to
the largest component) on the gradient; mixed path |dNLL| < 1e-3 absolute
and 1e-4 relative on the gradient.
"""
import numpy as np
import pytest

from ctpwa_b200 import workloads
from oracle.binding import Oracle

pytestmark = pytest.mark.gpu

SMALL = {"pipi_rho": (20_000, 5_000, 0), "pipi_3rho": (20_000, 5_000, 1_000), "kkpi": (20_000, 5_000, 1_000),
         "ksks": (20_000, 5_000, 0)}


@pytest.fixture(scope="module")
def setups(tmp_path_factory):
    import torch
    import ctpwa_b200

    out = {}
    for name, (nph, nda, nbk) in SMALL.items():
        d = tmp_path_factory.mktemp(name)
        cfg = workloads.make(name, d, n_phsp=nph, n_data=nda, n_bkg=nbk, accept_reject=False, seed=3)
        ana = ctpwa_b200.analysis(cfg)
        orc = Oracle(cfg)
        rng = np.random.default_rng(11)
        p = workloads.true_params(ana.getNVector(), ana.getFreeResParams()[0].numpy())
        p[2 * ana.getNVector():] *= 1 + 0.01 * rng.standard_normal(ana.getNFreeTheta())
        out[name] = (ana, orc, torch.tensor(p, dtype=torch.float64, device="cuda"), p)
    return out


@pytest.mark.parametrize("name", list(SMALL))
def test_counts_and_names_match_oracle(setups, name):
    ana, orc, _, _ = setups[name]
    assert ana.getNVector() == orc.nV
    assert ana.getNFreeTheta() == orc.nT
    assert ana.getNEvents() == orc.nev
    assert len(ana.getParamNames()) == ana.getNVector() + ana.getNFreeTheta()


@pytest.mark.parametrize("name", list(SMALL))
def test_fp64_nll_grad_parity(setups, name):
    ana, orc, pt, p = setups[name]
    nll, g = ana.getNLLAndGrad(pt, "fp64")
    onll, og, _ = orc.nll_grad(p)
    nll = float(nll)
    g = g.cpu().numpy()
    assert abs(nll - onll) <= 1e-10 * max(1.0, abs(onll)), (nll, onll)
    assert np.max(np.abs(g - og)) <= 1e-9 * np.max(np.abs(og)), (g, og)


@pytest.mark.parametrize("name", list(SMALL))
def test_mixed_nll_grad_close(setups, name):
    ana, orc, pt, p = setups[name]
    nll, g = ana.getNLLAndGrad(pt, "mixed")
    onll, og, _ = orc.nll_grad(p)
    assert abs(float(nll) - onll) < 1e-3
    assert np.max(np.abs(g.cpu().numpy() - og)) <= 1e-4 * np.max(np.abs(og))


@pytest.mark.parametrize("name", list(SMALL))
def test_intensity_parity(setups, name):
    ana, orc, pt, p = setups[name]
    for kind in (0, 1):
        f = ana.getIntensity(pt, kind).cpu().numpy()
        of = orc.intensity(kind, p)
        # per event, 1e-10 relative (the FP64 bar; symmetrised amplitudes can
        # cancel between their exchange terms, so single events sit above 1e-11)
        assert np.max(np.abs(f - of) / np.maximum(np.abs(of), 1e-300)) < 1e-10


def test_bitwise_reproducible(setups):
    ana, _, pt, _ = setups["kkpi"]
    a = ana.getNLLAndGrad(pt, "fp64")
    b = ana.getNLLAndGrad(pt, "fp64")
    assert float(a[0]) == float(b[0])
    assert bool((a[1] == b[1]).all())


def test_autograd_and_host_entry(setups):
    import torch

    ana, _, pt, p = setups["kkpi"]
    q = pt.clone().requires_grad_(True)
    nll = ana.getNLL(q)
    (g,) = torch.autograd.grad(nll, q)
    nll2, g2 = ana.getNLLAndGrad(pt, "fp64")
    assert float(nll) == float(nll2)
    assert bool((g == g2).all())
    hn, hg = ana.getNLLHost(p)
    assert hn == float(nll2)
    assert np.array_equal(hg, g2.cpu().numpy())


def test_param_checks(setups):
    import torch

    ana, _, pt, _ = setups["pipi_rho"]
    with pytest.raises(RuntimeError):
        ana.getNLL(pt.float())
    with pytest.raises(RuntimeError):
        ana.getNLL(pt.cpu())
    with pytest.raises(RuntimeError):
        ana.getNLL(pt[:-1])


@pytest.mark.parametrize("name", ["kkpi", "pipi_3rho"])
def test_mixed_unbiased_at_scale(tmp_path, name):
    """Mixed vs FP64 at 2M phase-space / 200k data events.

    The normalisation term is (W_data - W_bkg) log(mean f_phsp): a relative
    bias of the mixed form's phase-space mean of 3e-8 would already shift the
    NLL by ~6e-3 here, while unbiased per-event rounding stays near 1e-4."""
    import torch
    import ctpwa_b200

    cfg = workloads.make(name, tmp_path, n_phsp=2_000_000, n_data=200_000, n_bkg=20_000, accept_reject=False, seed=5)
    ana = ctpwa_b200.analysis(cfg)
    p = workloads.true_params(ana.getNVector(), ana.getFreeResParams()[0].numpy())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    n64, g64 = ana.getNLLAndGrad(pt, "fp64")
    nmx, gmx = ana.getNLLAndGrad(pt, "mixed")
    assert abs(float(n64) - float(nmx)) < 5e-4, (float(n64), float(nmx))
    assert float((g64 - gmx).abs().max()) <= 1e-4 * float(g64.abs().max())


def test_shard_sums_match_oracle_and_unsharded(tmp_path):
    """Device shard sums (multi-GPU exchange buffer) against the oracle's, and
    two shards combined against the unsharded evaluation."""
    import torch
    import ctpwa_b200

    cfg = workloads.make("kkpi", tmp_path, n_phsp=30_001, n_data=6_003, n_bkg=1_001, accept_reject=False, seed=12)
    full = ctpwa_b200.analysis(cfg)
    p = workloads.true_params(full.getNVector(), full.getFreeResParams()[0].numpy())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    shards = [ctpwa_b200.analysis(cfg, shard=(r, 2)) for r in range(2)]
    dev = [a.getShardSums(pt, "fp64") for a in shards]
    for r, s in enumerate(dev):
        os_ = Oracle(cfg, shard=(r, 2)).shard_sums(p)
        s = s.cpu().numpy()
        assert np.max(np.abs(s - os_)) <= 1e-10 * np.max(np.abs(os_)), r
    tot = dev[0] + dev[1]
    for prec in ("fp64", "mixed"):
        tot = shards[0].getShardSums(pt, prec) + shards[1].getShardSums(pt, prec)
        nll, g = shards[0].finalizeShardSums(pt, tot)
        n_ref, g_ref = full.getNLLAndGrad(pt, prec)
        tol = 1e-10 if prec == "fp64" else 1e-6
        assert abs(float(nll) - float(n_ref)) <= tol * max(1.0, abs(float(n_ref))), (prec, float(nll), float(n_ref))
        assert float((g - g_ref).abs().max()) <= tol * 10 * float(g_ref.abs().max()), prec


def test_hessian_matches_oracle_fd(setups):
    """Device Hessian (central differences of the exact device gradient) vs
    central differences of the oracle's dual-number gradient, same steps."""
    ana, orc, pt, p = setups["kkpi"]
    H = ana.getHessian(pt, method="fd").cpu().numpy()
    n = p.size
    Ho = np.zeros((n, n))
    for i in range(n):
        h = 1e-5 * max(abs(p[i]), 1e-2)
        q = p.copy()
        q[i] += h
        _, gp, _ = orc.nll_grad(q)
        q[i] -= 2 * h
        _, gm, _ = orc.nll_grad(q)
        Ho[i] = (gp - gm) / (2 * h)
    Ho = 0.5 * (Ho + Ho.T)
    assert np.allclose(H, H.T, rtol=0, atol=0)
    assert np.max(np.abs(H - Ho)) <= 1e-6 * np.max(np.abs(Ho)), np.max(np.abs(H - Ho)) / np.max(np.abs(Ho))


@pytest.mark.parametrize("name", ["kkpi", "pipi_3rho", "ksks"])
def test_exact_hessian_matches_oracle(setups, name):
    """Exact device Hessian (forward mode over the adjoint pass) vs
    Richardson-extrapolated differences of the oracle's exact gradient
    (accurate to ~2e-10 of the largest entry). The unsymmetrised rows H e_i
    come from independent dual-number passes and must already be symmetric
    to rounding."""
    import torch

    ana, orc, pt, p = setups[name]
    n = p.size
    rows = ana.getHessianVectorProduct(pt, torch.eye(n, dtype=torch.float64)).cpu().numpy()
    scale = np.max(np.abs(rows))
    assert np.max(np.abs(rows - rows.T)) <= 1e-11 * scale, np.max(np.abs(rows - rows.T)) / scale
    H = ana.getHessian(pt).cpu().numpy()
    assert np.array_equal(H, H.T)
    Ho = orc.hessian_fd(p)
    assert np.max(np.abs(H - Ho)) <= 1e-8 * scale, np.max(np.abs(H - Ho)) / scale
    # central differences of the device gradient (step 1e-5 relative) agree to
    # their own truncation error, a few 1e-6 of the largest entry
    Hfd = ana.getHessian(pt, method="fd").cpu().numpy()
    assert np.max(np.abs(H - Hfd)) <= 1e-5 * scale


def test_hessian_vector_products_linear(setups):
    """H u for arbitrary directions equals the full exact Hessian times u."""
    import torch

    ana, orc, pt, p = setups["kkpi"]
    rng = np.random.default_rng(5)
    U = rng.standard_normal((3, p.size))
    HU = ana.getHessianVectorProduct(pt, torch.tensor(U)).cpu().numpy()
    H = ana.getHessian(pt).cpu().numpy()
    ref = U @ H
    assert np.max(np.abs(HU - ref)) <= 1e-11 * np.max(np.abs(ref))
    one = ana.getHessianVectorProduct(pt, torch.tensor(U[1])).cpu().numpy()
    assert np.array_equal(one[0], HU[1])


def test_sharded_exact_hessian(tmp_path):
    """Two event shards: tangent sums vs the oracle's differentiated shard
    sums, the finalize vs the oracle's differentiated finalize, and the summed
    shards' Hessian vs the unsharded one."""
    import torch
    import ctpwa_b200

    cfg = workloads.make("kkpi", tmp_path, n_phsp=8_000, n_data=2_000, n_bkg=400, accept_reject=False, seed=5)
    full = ctpwa_b200.analysis(cfg)
    p = workloads.true_params(full.getNVector(), full.getFreeResParams()[0].numpy())
    p[2 * full.getNVector():] *= 1.002
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    n = p.size
    eye = torch.eye(n, dtype=torch.float64)
    shards = [ctpwa_b200.analysis(cfg, shard=(r, 2)) for r in range(2)]
    vs = [a.getShardSums(pt, "fp64") for a in shards]
    ts = [a.getShardHvpSums(pt, eye) for a in shards]
    rng = np.random.default_rng(2)
    U = rng.standard_normal((2, n))
    for r in range(2):
        o = Oracle(cfg, shard=(r, 2))
        t_dev = shards[r].getShardHvpSums(pt, torch.tensor(U)).cpu().numpy().reshape(2, -1)
        t_orc = o.hvp_sums_fd(p, U)
        assert np.max(np.abs(t_dev - t_orc)) <= 1e-8 * np.max(np.abs(t_orc)), r
    vsum, tsum = vs[0] + vs[1], ts[0] + ts[1]
    H = shards[0].finalizeShardHvp(pt, eye, vsum, tsum).cpu().numpy()
    Hf = full.getHessianVectorProduct(pt, eye).cpu().numpy()
    scale = np.max(np.abs(Hf))
    assert np.max(np.abs(H - Hf)) <= 1e-10 * scale
    orc = Oracle(cfg)
    Ho = orc.finalize_hvp_fd(p, np.eye(n), vsum.cpu().numpy(), tsum.cpu().numpy())
    assert np.max(np.abs(H - Ho)) <= 1e-8 * scale


def test_partial_integrals_and_fit_fractions(setups, tmp_path):
    """Partial-wave integrals vs the oracle's amplitude columns; fit fractions
    sum to one; phase-space truth sample read on demand."""
    import torch
    import ctpwa_b200

    ana, orc, pt, p = setups["pipi_3rho"]
    nV = ana.getNVector()
    I = ana.getPartialIntegrals(pt, 0).cpu().numpy()
    m = ana.getModel()
    cols = orc.columns(0, p[2 * nV:])  # [ev][pol][nA]
    chain, ratio = m["coupling"]["amp_chain"], m["coupling"]["ratio"]
    v = np.array([ratio[a] * complex(p[chain[a]], p[nV + chain[a]]) for a in range(cols.shape[2])])
    ref = []
    for b in m["blocks"]:
        nsl = len(m["groups"][b["group"]]["sl_combs"])
        S = np.einsum("epa,a->ep", cols[:, :, b["site"]:b["site"] + nsl], v[b["site"]:b["site"] + nsl])
        ref.append(np.sum(np.abs(S) ** 2))
    ref = np.array(ref)
    assert np.max(np.abs(I - ref)) <= 1e-10 * np.max(np.abs(ref))
    ff = ana.getFitFractions(pt)
    assert ff.shape == (ana.getNBlocks(), 2)
    assert abs(float(ff[:, 0].sum()) - 1.0) < 1e-12
    # a config with Data.phsp_truth integrates over that sample
    cfg = workloads.make("pipi_rho", tmp_path, n_phsp=5_000, n_data=1_000, n_bkg=0, accept_reject=False, seed=21)
    from ctpwa_b200 import toymc

    truth = toymc.phase_space(workloads.M_JPSI, workloads.MASSES["pipi_rho"], 7_000, 77)
    toymc.write_npy(tmp_path / "truth.npy", truth)
    text = open(cfg).read().replace("Data:\n", f'Data:\n  phsp_truth: [npy, "{tmp_path / "truth.npy"}"]\n', 1)
    open(cfg, "w").write(text)
    a2 = ctpwa_b200.analysis(cfg)
    q = torch.tensor(workloads.true_params(a2.getNVector(), a2.getFreeResParams()[0].numpy()), dtype=torch.float64,
                     device="cuda")
    assert float(a2.getPartialIntegrals(q, 3).sum()) > 0
    assert abs(float(a2.getFitFractions(q)[:, 0].sum()) - 1.0) < 1e-12


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_staged_tables_match_direct_loads(tmp_path, monkeypatch, mode):
    """The fused kernels with the event tables streamed through shared memory
    (CTPWA_STAGE=1: frontier rows by per-warp bulk copies; 2: frontier and
    angular rows; 3: frontier values by per-thread asynchronous copies) give
    the same results as with direct loads."""
    import torch
    import ctpwa_b200

    cfg = workloads.make("kkpi", tmp_path, n_phsp=70_001, n_data=9_999, n_bkg=777, accept_reject=False, seed=31)
    # the same launch shape for both handles (room for the buffers), so every
    # thread sums the same events in the same order
    monkeypatch.setenv("CTPWA_F64_ACC_SMEM", "0")
    monkeypatch.setenv("CTPWA_STAGE", "0")
    if mode == 2:
        # full tables in both handles: at one CTA per SM the unstaged kernel
        # still fits two, the staged one with the angular rows only one
        monkeypatch.setenv("CTPWA_NO_POL_PAIRING", "1")
        monkeypatch.setenv("CTPWA_F64_MINB", "1")
        monkeypatch.setenv("CTPWA_MX_MINB", "1")
    direct = ctpwa_b200.analysis(cfg)
    p = workloads.true_params(direct.getNVector(), direct.getFreeResParams()[0].numpy())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    monkeypatch.setenv("CTPWA_STAGE", str(mode))
    staged = ctpwa_b200.analysis(cfg)
    shape = staged.launchShape()
    assert shape["fp64"]["stage"] == mode and shape["mixed"]["stage"] == mode, shape
    assert direct.launchShape()["mixed"]["stage"] == 0
    assert direct.launchShape()["mixed"]["grid"] == shape["mixed"]["grid"]
    for prec in ("fp64", "mixed"):
        n0, g0 = direct.getNLLAndGrad(pt, prec)
        n1, g1 = staged.getNLLAndGrad(pt, prec)
        assert abs(float(n0) - float(n1)) <= 1e-12 * abs(float(n0)), prec
        assert float((g0 - g1).abs().max()) <= 1e-10 * float(g0.abs().max()), prec


def test_write_result_export(setups, tmp_path):
    """writeResult: per-event totals and block weights from the device export
    against the oracle's amplitude columns; interference diagonal = 2 x block
    integrals; total weights sum to the data yield."""
    ana, orc, pt, p = setups["kkpi"]
    out = ana.writeResult(pt, str(tmp_path / "res.npz"), is_saved_weight=1)
    nV = ana.getNVector()
    m = ana.getModel()
    cols = orc.columns(0, p[2 * nV:])
    chain, ratio = m["coupling"]["amp_chain"], m["coupling"]["ratio"]
    v = np.array([ratio[a] * complex(p[chain[a]], p[nV + chain[a]]) for a in range(cols.shape[2])])
    S = np.einsum("epa,a->ep", cols, v)
    tot = np.sum(np.abs(S) ** 2, axis=1)
    assert np.max(np.abs(out["totalweight"] / out["norm_factor"] - tot) / tot) < 1e-10
    assert abs(out["totalweight"].sum() - out["data_integral"]) < 1e-8 * out["data_integral"]
    I = ana.getPartialIntegrals(pt, 0).cpu().numpy()
    assert np.allclose(np.diag(out["interference"]), 2 * I, rtol=1e-10)
    for i in range(ana.getNBlocks()):
        assert abs(out[f"weight_{i}"].sum() / out["norm_factor"] - I[i]) <= 1e-10 * I[i]
    loaded = np.load(tmp_path / "res.npz")
    assert set(loaded.files) >= {"legends", "interference", "totalweight"}


def test_in_memory_samples_match_files(tmp_path):
    """analysis.from_device over the same events as a file-based analysis
    gives bit-identical results; the on-device toy generator is seeded."""
    import torch
    import ctpwa_b200
    from ctpwa_b200 import toymc

    cfg = workloads.make("kkpi", tmp_path, n_phsp=30_001, n_data=4_001, n_bkg=999, accept_reject=False, seed=21)
    files = ctpwa_b200.analysis(cfg)
    dev = [torch.from_numpy(np.load(tmp_path / f)).cuda() for f in ("phsp.npy", "data.npy", "bkg.npy")]
    w = [None, None, torch.full((dev[2].shape[0],), 0.3, dtype=torch.float64, device="cuda")]
    mem = ctpwa_b200.analysis.from_device(cfg, dev[0], dev[1], dev[2], weights=w)
    assert tuple(mem.getNEvents()) == tuple(files.getNEvents())
    p = workloads.true_params(files.getNVector(), files.getFreeResParams()[0].numpy())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    for prec in ("fp64", "mixed"):
        n0, g0 = files.getNLLAndGrad(pt, prec)
        n1, g1 = mem.getNLLAndGrad(pt, prec)
        assert float(n0) == float(n1) and torch.equal(g0, g1), prec
    c1, ph1, d1 = workloads.make_device("pipi_rho", tmp_path / "a", 50_000, 5_000, seed=4)
    c2, ph2, d2 = workloads.make_device("pipi_rho", tmp_path / "b", 50_000, 5_000, seed=4)
    assert ph1.shape == (50_000, 3, 4) and d1.shape == (5_000, 3, 4)
    assert torch.equal(ph1, ph2) and torch.equal(d1, d2)
    # accept-reject favours the resonance: data are not flat phase space
    flat = torch.from_numpy(toymc.phase_space(workloads.M_JPSI, workloads.MASSES["pipi_rho"], 5_000, 3))
    def m12(x):
        s = x[:, 0] + x[:, 1]
        return torch.sqrt(s[:, 0] ** 2 - (s[:, 1:] ** 2).sum(1))
    near = lambda m: float(((m > 0.65) & (m < 0.9)).double().mean())
    assert near(m12(d1.cpu())) > 1.5 * near(m12(flat))


def test_device_phase_space_generator():
    """The CUDA phase-space generator: on-shell masses, momentum balance, flat
    Dalitz density, event i a function of (seed, i) only."""
    import torch
    from ctpwa_b200 import toymc

    M, masses = workloads.M_JPSI, (0.13975, 0.13975, 0.13495)
    p = toymc.phase_space_device(M, masses, 200_000, 9).cpu().numpy()
    m2 = p[..., 0] ** 2 - np.sum(p[..., 1:] ** 2, axis=-1)
    assert np.allclose(np.sqrt(np.maximum(m2, 0)), np.array(masses)[None, :], rtol=1e-9)
    tot = p.sum(axis=1)
    assert np.allclose(tot[:, 0], M, rtol=1e-12) and np.allclose(tot[:, 1:], 0.0, atol=1e-12)
    s12 = p[:, 0] + p[:, 1]
    s12 = s12[:, 0] ** 2 - np.sum(s12[:, 1:] ** 2, axis=1)
    s13 = p[:, 0] + p[:, 2]
    s13 = s13[:, 0] ** 2 - np.sum(s13[:, 1:] ** 2, axis=1)
    sel = (s12 > 2.0) & (s12 < 2.5)
    h, _ = np.histogram(s13[sel], bins=10)
    assert h[2:-2].std() / h[2:-2].mean() < 0.05
    a = toymc.phase_space_device(M, masses, 1_000, 5)
    b = toymc.phase_space_device(M, masses, 3_000, 5)
    assert torch.equal(a, b[:1_000])
    assert not torch.equal(a, toymc.phase_space_device(M, masses, 1_000, 6))


def test_polarisation_pairing(tmp_path, monkeypatch):
    """J/psi -> K+K-pi0: the M = +1 and M = -1 angular values are complex
    conjugates on every event, so the fused kernels store two of the three
    polarisations; results agree with those of the full tables."""
    import torch
    import ctpwa_b200

    cfg = workloads.make("kkpi", tmp_path, n_phsp=40_001, n_data=6_001, n_bkg=1_001, accept_reject=False, seed=33)
    paired = ctpwa_b200.analysis(cfg)
    shape = paired.launchShape()
    assert shape["fp64"]["pol_paired"] == 1 and shape["mixed"]["pol_paired"] == 1
    monkeypatch.setenv("CTPWA_NO_POL_PAIRING", "1")
    full = ctpwa_b200.analysis(cfg)
    assert full.launchShape()["mixed"]["pol_paired"] == 0
    p = workloads.true_params(full.getNVector(), full.getFreeResParams()[0].numpy())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    n0, g0 = full.getNLLAndGrad(pt, "fp64")
    n1, g1 = paired.getNLLAndGrad(pt, "fp64")
    assert abs(float(n0) - float(n1)) <= 1e-12 * abs(float(n0))
    assert float((g0 - g1).abs().max()) <= 1e-10 * float(g0.abs().max())
    m0, h0 = full.getNLLAndGrad(pt, "mixed")
    m1, h1 = paired.getNLLAndGrad(pt, "mixed")
    # the paired form shares each conjugate pair's products, so the FP32
    # roundings differ from the full tables' (well below the 1e-3 bar)
    assert abs(float(m0) - float(m1)) < 1e-4
    assert float((h0 - h1).abs().max()) <= 1e-5 * float(h0.abs().max())
    orc = Oracle(cfg)
    onll, og, _ = orc.nll_grad(p)
    assert abs(float(n1) - onll) <= 1e-10 * abs(onll)


def _weighted_config(tmp_path, n_phsp, n_data, n_bkg, seed, short_bkg=False):
    """kkpi config with per-event weight files for data, phase space and
    background (.dat, one value per event; with short_bkg the background file
    lists fewer values than events, which the reader pads with zeros)."""
    cfg = workloads.make("kkpi", tmp_path, n_phsp=n_phsp, n_data=n_data, n_bkg=n_bkg, accept_reject=False, seed=seed,
                         gpu_generator=False)
    rng = np.random.default_rng(seed + 100)
    lines = []
    for key, n, lo, hi in (("data_weights", n_data, 0.5, 1.5), ("phsp_weights", n_phsp, 0.8, 1.2),
                           ("bkg_weights", n_bkg - 3 if short_bkg else n_bkg, 0.1, 0.5)):
        if n <= 0 and key == "bkg_weights" and n_bkg == 0:
            continue
        f = tmp_path / f"{key}.dat"
        np.savetxt(f, rng.uniform(lo, hi, max(n, 0)))
        lines.append(f'  {key}: [dat, "{f}"]')
    text = open(cfg).read()
    text = "\n".join(l for l in text.splitlines() if not l.strip().startswith("bkg_weights:"))
    text = text.replace("Data:\n", "Data:\n" + "\n".join(lines) + "\n", 1)
    open(cfg, "w").write(text + "\n")
    return cfg


@pytest.mark.parametrize("short_bkg", [False, True])
def test_per_event_weight_files(tmp_path, short_bkg):
    """Per-event weights from .dat files for data, phase space (weighted
    normalisation) and background, against the oracle reading the same
    files; a background weight file shorter than the sample is padded with
    zeros as the reference's reader does."""
    import torch
    import ctpwa_b200

    cfg = _weighted_config(tmp_path, 20_011, 3_001, 507, seed=41, short_bkg=short_bkg)
    ana = ctpwa_b200.analysis(cfg)
    orc = Oracle(cfg)
    p = workloads.true_params(ana.getNVector(), ana.getFreeResParams()[0].numpy())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    onll, og, _ = orc.nll_grad(p)
    nll, g = ana.getNLLAndGrad(pt, "fp64")
    assert abs(float(nll) - onll) <= 1e-10 * max(1.0, abs(onll)), (float(nll), onll)
    assert np.max(np.abs(g.cpu().numpy() - og)) <= 1e-9 * np.max(np.abs(og))
    nmx, gmx = ana.getNLLAndGrad(pt, "mixed")
    assert abs(float(nmx) - onll) < 1e-3
    assert np.max(np.abs(gmx.cpu().numpy() - og)) <= 1e-4 * np.max(np.abs(og))


@pytest.mark.parametrize("sizes", [(1, 1, 0), (33, 5, 1), (257, 31, 2), (1000, 1, 0)])
def test_tiny_and_ragged_samples(tmp_path, sizes):
    """Samples of one event and sizes off every tile boundary: FP64 against
    the oracle, the mixed form within its bar, the exact Hessian symmetric."""
    import torch
    import ctpwa_b200

    n_phsp, n_data, n_bkg = sizes
    cfg = workloads.make("kkpi", tmp_path, n_phsp=n_phsp, n_data=n_data, n_bkg=n_bkg, accept_reject=False, seed=43,
                         gpu_generator=False)
    ana = ctpwa_b200.analysis(cfg)
    orc = Oracle(cfg)
    assert ana.getNEvents() == orc.nev
    p = workloads.true_params(ana.getNVector(), ana.getFreeResParams()[0].numpy())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    onll, og, _ = orc.nll_grad(p)
    nll, g = ana.getNLLAndGrad(pt, "fp64")
    assert abs(float(nll) - onll) <= 1e-10 * max(1.0, abs(onll)), (float(nll), onll)
    assert np.max(np.abs(g.cpu().numpy() - og)) <= 1e-9 * max(1e-300, np.max(np.abs(og)))
    nmx, _ = ana.getNLLAndGrad(pt, "mixed")
    assert abs(float(nmx) - onll) < 1e-3
    H = ana.getHessian(pt).cpu().numpy()
    assert np.all(np.isfinite(H))
    assert np.max(np.abs(H - H.T)) <= 1e-9 * max(1e-300, np.max(np.abs(H)))


def _features_config(tmp_path, n_phsp=20_011, n_data=3_001):
    """tests/golden/features.yml (trans folding, var_range, gauss_constr,
    fix_var, a multi-mode intermediate, an expanded chain) over seeded
    K+ K- eta phase-space samples written next to it."""
    import os
    import shutil

    from ctpwa_b200 import toymc

    here = os.path.dirname(os.path.abspath(__file__))
    cfg = tmp_path / "config.yml"
    shutil.copy(os.path.join(here, "golden", "features.yml"), cfg)
    masses = [0.493677, 0.493677, 0.547862]
    toymc.write_npy(tmp_path / "phsp.npy", toymc.phase_space(3.0969, masses, n_phsp, 51))
    toymc.write_npy(tmp_path / "data.npy", toymc.phase_space(3.0969, masses, n_data, 52))
    return str(cfg)


def test_feature_config_parity(tmp_path, monkeypatch):
    """The feature config evaluated on the device against the oracle: FP64
    NLL and gradient (folded couplings, Gaussian constraint, fixed and
    range-limited parameters), the mixed form, and the exact Hessian against
    Richardson differences of the oracle's gradient."""
    import torch
    import ctpwa_b200

    monkeypatch.chdir(tmp_path)  # the config names its samples relative to its directory
    cfg = _features_config(tmp_path)
    ana = ctpwa_b200.analysis(cfg)
    assert ana.isValid()
    orc = Oracle(cfg)
    assert ana.getNVector() == orc.nV and ana.getNFreeTheta() == orc.nT
    p = workloads.true_params(ana.getNVector(), ana.getFreeResParams()[0].numpy())
    rng = np.random.default_rng(9)
    p[2 * ana.getNVector():] *= 1 + 0.01 * rng.standard_normal(ana.getNFreeTheta())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    onll, og, _ = orc.nll_grad(p)
    nll, g = ana.getNLLAndGrad(pt, "fp64")
    assert abs(float(nll) - onll) <= 1e-10 * max(1.0, abs(onll)), (float(nll), onll)
    assert np.max(np.abs(g.cpu().numpy() - og)) <= 1e-9 * np.max(np.abs(og))
    nmx, gmx = ana.getNLLAndGrad(pt, "mixed")
    assert abs(float(nmx) - onll) < 1e-3
    assert np.max(np.abs(gmx.cpu().numpy() - og)) <= 1e-4 * np.max(np.abs(og))
    H = ana.getHessian(pt).cpu().numpy()
    Ho = orc.hessian_fd(p)
    assert np.max(np.abs(H - Ho)) <= 1e-6 * np.max(np.abs(Ho)), np.max(np.abs(H - Ho)) / np.max(np.abs(Ho))


_SHAPES = {
    "bw_gs_hist_flatte": """Resonances:
  Kst892:    {J: 1, P: -1, model: BW, parameters: [0.8955, 0.047], free: [0, 1]}
  Kst1410:   {J: 1, P: -1, model: GS, parameters: [1.414, 0.232], free: [0, 1]}
  Kst2_1430: {J: 2, P: 1, model: Hist, file: "@DIR@/hist.dat", bins: 40, range: [0.6, 2.7]}
  X1680: {J: 1, P: -1, model: Flatte, parameters: [1.68, 0.3, 0.1], free: [0, 1, 2], channels: [[0.493677, 0.493677], [0.13957, 0.13957]]}
""",
    "interp": """Resonances:
  Kst892:    {J: 1, P: -1, model: BWR, parameters: [0.8955, 0.047], free: [0, 1]}
  Kst1410:   {J: 1, P: -1, model: Interp, file: "@DIR@/interp.dat"}
  Kst2_1430: {J: 2, P: 1, model: BWR, parameters: [1.4256, 0.0985], free: [0, 1]}
  X1680: {J: 1, P: -1, model: BWR, parameters: [1.68, 0.15], free: [0, 1]}
""",
}


def _shapes_config(tmp_path, variant):
    """K+K-pi0 chains with the other built-in lineshapes: BW, GS, a histogram
    (Hist), Flatte with channels, a complex interpolation table (Interp)."""
    cfg = workloads.make("kkpi", tmp_path, n_phsp=20_011, n_data=3_001, n_bkg=0, accept_reject=False, seed=61,
                         gpu_generator=False)
    x = np.linspace(0.6, 2.7, 40)
    np.savetxt(tmp_path / "hist.dat", 1.0 + 0.5 * np.sin(3 * x))
    xi = np.linspace(0.55, 2.75, 60)
    np.savetxt(tmp_path / "interp.dat", np.c_[xi, np.cos(2 * xi) / (1 + xi), np.sin(xi) / (1 + xi)])
    text = open(cfg).read()
    text = text[:text.index("Resonances:")] + _SHAPES[variant].replace("@DIR@", str(tmp_path))
    open(cfg, "w").write(text)
    return cfg


@pytest.mark.parametrize("variant", list(_SHAPES))
def test_builtin_lineshapes_parity(tmp_path, variant):
    """BW, GS, Hist, Flatte and Interp lineshapes in the fused kernels: FP64
    NLL and gradient against the oracle, the mixed form within its bar."""
    import torch
    import ctpwa_b200

    cfg = _shapes_config(tmp_path, variant)
    ana = ctpwa_b200.analysis(cfg)
    assert ana.isValid()
    orc = Oracle(cfg)
    assert ana.getNVector() == orc.nV and ana.getNFreeTheta() == orc.nT
    p = workloads.true_params(ana.getNVector(), ana.getFreeResParams()[0].numpy())
    p[2 * ana.getNVector():] *= 1 + 0.01 * np.random.default_rng(3).standard_normal(ana.getNFreeTheta())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    onll, og, _ = orc.nll_grad(p)
    nll, g = ana.getNLLAndGrad(pt, "fp64")
    assert abs(float(nll) - onll) <= 1e-10 * max(1.0, abs(onll)), (float(nll), onll)
    assert np.max(np.abs(g.cpu().numpy() - og)) <= 1e-9 * np.max(np.abs(og))
    nmx, gmx = ana.getNLLAndGrad(pt, "mixed")
    assert abs(float(nmx) - onll) < 1e-3
    assert np.max(np.abs(gmx.cpu().numpy() - og)) <= 1e-4 * np.max(np.abs(og))
    H = ana.getHessian(pt).cpu().numpy()
    assert np.max(np.abs(H - H.T)) <= 1e-9 * np.max(np.abs(H))


_EXPRS = [
    # signs, right-associative powers and the imaginary unit
    "-mass^2^0.5 + (m/gKK)^(1j*gKK) - -gpipi + 2^-1^2*m + 3*-m/mass^2",
    # builtin lineshapes inside an expression, q0 with and without arguments
    "BWR(mass, gKK, 1, 3.0) * Bf(1, q, q0(m), 3.0) + gpipi*exp(1j*m) * q0",
    # one-argument functions and nested parentheses
    "mass^2/(mass^2 - m^2 - 1j*mass*gKK) * (1 + gpipi*Re(conj(1j*m)) + abs(gpipi - 1j)/sqrt(m) - Im(ln(m*gKK)))",
    # constant folding and signed zeros on the branch cut of log / pow (the conjugate branch if either were lost)
    "BWR(mass, gKK) * ((-m)^0.5 * (m*-2)^gpipi + log(-gKK*m) + exp(-m)*(-1)^gpipi)",
    "BWR(mass, gKK) * ((-mass - m)^1.5 + conj(-m)^0.3 - (m/-1)^0.5 + (-1*m)^0.5 + sin(-mass)^2.5 * cos(mass)^0.5)",
    "BWR(mass, gKK) * (0^(m-2) + mass^1*gpipi^1 + 1^m + (0-m)^0.5 - -(-m)^0.5 + (-(m^2-mass^2))^gpipi)",
]


@pytest.mark.parametrize("expr", _EXPRS)
def test_custom_expression_language_parity(tmp_path, expr):
    """The custom-lineshape language through the code generator: precedence,
    signs, the imaginary unit and builtin calls, FP64 NLL and gradient against
    the oracle, whose evaluator is pinned to the reference's compiled one."""
    import torch
    import ctpwa_b200

    cfg = workloads.make("kkpi", tmp_path, n_phsp=8_000, n_data=2_000, n_bkg=0, accept_reject=False, seed=71,
                         gpu_generator=False)
    text = open(cfg).read()
    old = 'expr: "Flatte(mass, gKK, gpipi, 0.493677, 0.493677, 0.13957, 0.13957) * Bf(1, q, q0, 3.0)"'
    assert old in text
    open(cfg, "w").write(text.replace(old, f'expr: "{expr}"'))
    ana = ctpwa_b200.analysis(cfg)
    assert ana.isValid()
    orc = Oracle(cfg)
    p = workloads.true_params(ana.getNVector(), ana.getFreeResParams()[0].numpy())
    p[2 * ana.getNVector():] *= 1 + 0.01 * np.random.default_rng(5).standard_normal(ana.getNFreeTheta())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    onll, og, _ = orc.nll_grad(p)
    nll, g = ana.getNLLAndGrad(pt, "fp64")
    assert abs(float(nll) - onll) <= 1e-10 * max(1.0, abs(onll)), (float(nll), onll)
    assert np.max(np.abs(g.cpu().numpy() - og)) <= 1e-9 * np.max(np.abs(og))


def test_device_covariance(setups):
    """Covariance on the device: the FP64 inverse of the Hessian over the free
    parameters equals the host inverse; a matrix that is not positive
    definite is reported. The sample here is not drawn from the model, so its
    Hessian at this point need not be positive definite; the inverse is
    checked on the Hessian shifted to a well-conditioned SPD matrix."""
    import torch
    import ctpwa_b200

    ana, _, pt, _ = setups["kkpi"]
    H = ana.getHessian(pt)
    n = ana.getNVector()
    free = [j for j in range(ana.getNParams()) if j not in (0, n)]
    Hf = H.cpu().numpy()[np.ix_(free, free)]
    ev = np.linalg.eigvalsh(Hf)
    if ev[0] <= 0.0:
        with pytest.raises(RuntimeError, match="not positive definite"):
            ana.getCovariance(pt, hessian=H)
    shift = max(0.0, -ev[0]) + 0.1 * np.max(np.abs(ev))
    Hs = H + shift * torch.eye(H.shape[0], dtype=torch.float64, device=H.device)
    C = ana.getCovariance(pt, hessian=Hs).cpu().numpy()
    ref = np.linalg.inv(Hf + shift * np.eye(len(free)))
    assert np.max(np.abs(C[np.ix_(free, free)] - ref)) <= 1e-9 * np.max(np.abs(ref))
    assert np.all(C[0] == 0) and np.all(C[:, n] == 0)
    with pytest.raises(RuntimeError, match="not positive definite"):
        ctpwa_b200.spd_inverse(-torch.eye(4, dtype=torch.float64, device="cuda"))


def test_dat_momenta_match_npy(tmp_path):
    """The .dat momenta reader (E px py pz per line, one line per final-state
    particle in Data.order, src/Analysis.cu:58-176): a handle on .dat copies
    of the samples (17 significant digits) equals the handle on the .npy
    originals bit for bit."""
    import torch
    import ctpwa_b200
    from oracle import refcuda

    cfg = workloads.make("kkpi", tmp_path, n_phsp=20_011, n_data=3_001, n_bkg=503, accept_reject=False, seed=19)
    dcfg = refcuda.dat_config(cfg, tmp_path / "dat")
    a, b = ctpwa_b200.analysis(cfg), ctpwa_b200.analysis(dcfg)
    assert a.getNEvents() == b.getNEvents()
    p = workloads.true_params(a.getNVector(), a.getFreeResParams()[0].numpy())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    for prec in ("fp64", "mixed"):
        na, ga = a.getNLLAndGrad(pt, prec)
        nb, gb = b.getNLLAndGrad(pt, prec)
        assert float(na) == float(nb) and torch.equal(ga, gb)


def test_fp64_only_handles(tmp_path):
    """Handles created without the mixed-form tables and the polarisation
    pairing (ctpwa_create_from_device_flags, CTPWA_CREATE_FP64_ONLY; the toy
    generator's accept-reject candidates): the same intensities bit for bit,
    FP64 NLL and gradient within 1e-12, and a clear error for the mixed form."""
    import torch
    import ctpwa_b200

    cfg = workloads.make("kkpi", tmp_path, n_phsp=30_001, n_data=4_001, n_bkg=999, accept_reject=False, seed=22)
    dev = [torch.from_numpy(np.load(tmp_path / f)).cuda() for f in ("phsp.npy", "data.npy", "bkg.npy")]
    full = ctpwa_b200.analysis.from_device(cfg, dev[0], dev[1], dev[2])
    lean = ctpwa_b200.analysis.from_device(cfg, dev[0], dev[1], dev[2], fp64_only=True)
    assert full.launchShape()["fp64"]["pol_paired"] == 1 and lean.launchShape()["fp64"]["pol_paired"] == 0
    assert lean.deviceBytes() < full.deviceBytes()
    p = workloads.true_params(full.getNVector(), full.getFreeResParams()[0].numpy())
    pt = torch.tensor(p, dtype=torch.float64, device="cuda")
    assert torch.equal(full.getIntensity(pt, kind=1), lean.getIntensity(pt, kind=1))
    n0, g0 = full.getNLLAndGrad(pt, "fp64")
    n1, g1 = lean.getNLLAndGrad(pt, "fp64")
    assert abs(float(n1) - float(n0)) <= 1e-12 * abs(float(n0))
    assert float((g1 - g0).abs().max()) <= 1e-11 * float(g0.abs().max())
    with pytest.raises(RuntimeError, match="mixed-precision tables"):
        lean.getNLLAndGrad(pt, "mixed")
