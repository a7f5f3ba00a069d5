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
