"""Fit-job serving loop: stream generation, admission bookkeeping (CPU) and,
on the GPU, that every job's result is the same alone and in the mix."""
import numpy as np
import pytest

from ctpwa_b200 import serving


def test_poisson_stream_is_seeded_and_bounded():
    a = serving.poisson_stream(5.0, 200, nd_range=(10_000, 2_000_000), seed=3)
    b = serving.poisson_stream(5.0, 200, nd_range=(10_000, 2_000_000), seed=3)
    assert [(j.arrival, j.n_data, j.model) for j in a] == [(j.arrival, j.n_data, j.model) for j in b]
    nd = np.array([j.n_data for j in a])
    assert nd.min() >= 10_000 and nd.max() <= 2_000_000
    assert all(j.n_phsp == 10 * j.n_data for j in a)
    arr = np.array([j.arrival for j in a])
    assert np.all(np.diff(arr) > 0)
    assert 0.5 / 5.0 < np.mean(np.diff(arr)) < 2.0 / 5.0  # mean inter-arrival 1/rate
    assert {j.model for j in a} == {"pipi_rho", "pipi_3rho"}


def test_admission_budget_accounting():
    srv = serving.Server.__new__(serving.Server)  # no GPU: only the bookkeeping
    import threading

    srv._lock = threading.Lock()
    srv._in_use = 0
    srv.budget = 1000
    assert srv.try_reserve(600)
    assert not srv.try_reserve(500)
    assert srv.try_reserve(400)
    srv.release(600)
    assert srv.try_reserve(500)
    assert srv._in_use == 900


def test_summary_percentiles():
    rs = []
    for j in range(4):
        r = serving.JobResult(job_id=j, model="pipi_rho", n_data=1, n_phsp=10, precision="mixed",
                              arrival=0.0, admitted=0.1 * j, finished=1.0 + j)
        r.eval_ms = [1.0, 2.0, 3.0]
        rs.append(r)
    rs.append(serving.JobResult(job_id=9, model="pipi_rho", n_data=1, n_phsp=10, precision="mixed", error="x"))
    s = serving.summary(rs, wall_s=3600.0)
    assert s["jobs"] == 5 and s["failed"] == 1 and s["fits_per_hour"] == 4.0
    assert s["eval_ms_p50"] == 2.0
    assert abs(s["fit_ms_p50"] - 2500.0) < 1e-9


@pytest.mark.gpu
def test_results_same_alone_and_in_the_mix():
    jobs = [serving.JobSpec(job_id=0, model="pipi_rho", n_data=8_000, n_phsp=80_000, seed=11, max_evals=25),
            serving.JobSpec(job_id=1, model="pipi_3rho", n_data=5_000, n_phsp=50_000, seed=12, max_evals=25),
            serving.JobSpec(job_id=2, model="pipi_rho", n_data=20_000, n_phsp=200_000, seed=13, max_evals=25,
                            precision="fp64")]
    alone = []
    srv = serving.Server(slots=1)
    try:
        for j in jobs:
            alone += srv.run([j], realtime=False)
    finally:
        srv.close()
    srv = serving.Server(slots=3)
    try:
        mixed = srv.run(jobs, realtime=False)
    finally:
        srv.close()
    for a, m in zip(alone, mixed):
        assert a.error is None and m.error is None, (a.error, m.error)
        assert a.n_evals == m.n_evals > 0
        assert abs(a.nll - m.nll) <= 1e-12 * abs(a.nll), (a.job_id, a.nll, m.nll)
        assert np.allclose(a.params, m.params, rtol=1e-12, atol=0)
        assert np.allclose(a.hessian, m.hessian, rtol=1e-10, atol=1e-10 * np.max(np.abs(a.hessian)))


@pytest.mark.gpu
def test_native_fit_reaches_the_scipy_minimum(tmp_path):
    """analysis.fit (projected L-BFGS in native code) from a perturbed start
    ends at the minimum scipy's L-BFGS-B finds over the same host-buffer
    evaluations, with every evaluation inside the resonance bounds."""
    import numpy as np
    from scipy.optimize import minimize

    import ctpwa_b200
    from ctpwa_b200 import workloads

    cfg = workloads.make("pipi_3rho", tmp_path, n_phsp=60_000, n_data=6_000, n_bkg=0, seed=21)
    ana = ctpwa_b200.analysis(cfg, precision="fp64")
    nV = ana.getNVector()
    res = ana.getFreeResParams().numpy()
    start = workloads.true_params(nV, res[0])
    rng = np.random.default_rng(5)
    start[1:nV] *= 1 + 0.1 * rng.standard_normal(nV - 1)
    start[nV + 1:2 * nV] *= 1 + 0.1 * rng.standard_normal(nV - 1)
    start[2 * nV:] *= 1 + 0.003 * rng.standard_normal(start.size - 2 * nV)
    x, nll, ne, it, status, lat = ana.fit(start, max_evals=300)
    assert status in (0, 1) and ne <= 300 and len(lat) == ne
    assert np.all(x[2 * nV:] >= res[1]) and np.all(x[2 * nV:] <= res[2])
    assert x[0] == start[0] and x[nV] == start[nV]
    assert abs(ana.getNLLHost(x)[0] - nll) == 0.0

    free = np.ones(start.size, dtype=bool)
    free[0] = free[nV] = False
    bounds = [(None, None)] * (2 * nV) + [(float(lo), float(hi)) for lo, hi in zip(res[1], res[2])]
    xf = start.copy()

    def fun(v):
        xf[free] = v
        f, g = ana.getNLLHost(xf)
        return f, g[free]

    ref = minimize(fun, start[free], jac=True, method="L-BFGS-B", bounds=[b for b, f in zip(bounds, free) if f],
                   options={"maxfun": 300, "maxcor": 20, "ftol": 1e-13, "gtol": 1e-9})
    assert nll <= ref.fun + 1e-6 * max(1.0, abs(ref.fun)), (nll, ref.fun)
    assert abs(nll - ref.fun) <= 1e-5 * max(1.0, abs(ref.fun)), (nll, ref.fun)


@pytest.mark.gpu
def test_profile_scan_is_parabolic_near_the_minimum():
    """Profile-likelihood scan (the other parameters refitted at each point):
    at the fitted value +- 1 and 2 sigma (sigma from the exact Hessian) the
    NLL rises by about s^2 / 2, and never falls below the best fit."""
    nV = 1  # pipi_rho: one coupling; parameter 2 is the rho mass, 3 its width
    jobs = [serving.JobSpec(job_id=0, model="pipi_rho", n_data=40_000, n_phsp=400_000, seed=31, max_evals=300,
                            precision="fp64", scan_param=2 * nV, scan_sigmas=(-2.0, -1.0, 1.0, 2.0)),
            serving.JobSpec(job_id=1, model="pipi_rho", n_data=40_000, n_phsp=400_000, seed=31, max_evals=300,
                            precision="fp64", scan_param=2 * nV + 1, scan_sigmas=(-1.0, 1.0))]
    srv = serving.Server(slots=2)
    try:
        res = srv.run(jobs, realtime=False)
    finally:
        srv.close()
    for r, spec in zip(res, jobs):
        assert r.error is None, r.error
        assert len(r.scan) == len(spec.scan_sigmas) and "scan" in r.phase_ms
        for (v, dnll), s in zip(r.scan, spec.scan_sigmas):
            assert dnll > -1e-6, (v, dnll)
            assert abs(dnll - 0.5 * s * s) <= 0.15 * s * s, (s, dnll)
        assert r.scan[0][0] < r.params[spec.scan_param] < r.scan[-1][0]


@pytest.mark.gpu
def test_multi_job_launch_equals_single_evaluations(tmp_path):
    """Several handles of one model evaluated in one launch per stage
    (ctpwa_nll_grad_multi): each job's NLL and gradient are those of its own
    evaluation, bit for bit, in both precisions; a handle of another model
    is rejected."""
    import torch
    import ctpwa_b200
    from ctpwa_b200 import workloads

    anas, params = [], []
    for k, (nph, nda, nbk) in enumerate([(30_011, 3_001, 0), (80_003, 8_009, 1_001), (12_007, 1_201, 0)]):
        cfg = workloads.make("pipi_3rho", tmp_path / f"j{k}", n_phsp=nph, n_data=nda, n_bkg=nbk,
                             accept_reject=False, seed=40 + k)
        a = ctpwa_b200.analysis(cfg)
        p = workloads.true_params(a.getNVector(), a.getFreeResParams()[0].numpy())
        p[2 * a.getNVector():] *= 1 + 0.01 * (k + 1)
        anas.append(a)
        params.append(torch.tensor(p, dtype=torch.float64, device="cuda"))
    b = ctpwa_b200.EvalBatch(0)
    try:
        for prec in ("fp64", "mixed"):
            for _ in range(2):  # the second call reuses the argument table
                res = b.nll_grad(anas, params, prec)
                torch.cuda.synchronize()
                for a, p, (n_m, g_m) in zip(anas, params, res):
                    n_s, g_s = a.getNLLAndGrad(p, prec)
                    assert float(n_m) == float(n_s) and torch.equal(g_m, g_s), prec
        other = ctpwa_b200.analysis(workloads.make("pipi_rho", tmp_path / "o", n_phsp=5_000, n_data=500, n_bkg=0,
                                                   accept_reject=False, seed=1))
        po = torch.tensor(workloads.true_params(other.getNVector(), other.getFreeResParams()[0].numpy()),
                          dtype=torch.float64, device="cuda")
        with pytest.raises(RuntimeError, match="one model"):
            b.nll_grad([anas[0], other], [params[0], po], "fp64")
    finally:
        b.close()


@pytest.mark.gpu
def test_batched_serving_same_results_and_shared_launches():
    """Serving with the fits' evaluations gathered into shared launches: each
    job's fitted parameters, NLL and Hessian equal those of the job run alone
    without batching, and the batch served several requests per round."""
    jobs = [serving.JobSpec(job_id=0, model="pipi_rho", n_data=8_000, n_phsp=80_000, seed=11, max_evals=25),
            serving.JobSpec(job_id=1, model="pipi_rho", n_data=12_000, n_phsp=120_000, seed=14, max_evals=25),
            serving.JobSpec(job_id=2, model="pipi_3rho", n_data=5_000, n_phsp=50_000, seed=12, max_evals=25),
            serving.JobSpec(job_id=3, model="pipi_3rho", n_data=6_000, n_phsp=60_000, seed=15, max_evals=25,
                            precision="fp64")]
    alone = []
    srv = serving.Server(slots=1)
    try:
        for j in jobs:
            alone += srv.run([j], realtime=False)
    finally:
        srv.close()
    srv = serving.Server(slots=4, batch=True)
    try:
        mixed = srv.run(jobs, realtime=False)
        rounds, requests = srv.batch.stats()
    finally:
        srv.close()
    for a, m in zip(alone, mixed):
        assert a.error is None and m.error is None, (a.error, m.error)
        assert a.n_evals == m.n_evals > 0
        assert a.nll == m.nll, (a.job_id, a.nll, m.nll)
        assert np.array_equal(a.params, m.params)
        assert np.allclose(a.hessian, m.hessian, rtol=1e-10, atol=1e-10 * np.max(np.abs(a.hessian)))
    assert requests == sum(m.n_evals for m in mixed)
    assert rounds < requests
