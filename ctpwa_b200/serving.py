"""Fit-job serving loop: toy-MC fits of uneven size sharing one GPU.

The workload pattern of the reference's fit driver (example/fit.py:115-216,
600-650) as a service: jobs arrive over time (a Poisson stream), each brings
its own seeded event sample (data by accept-reject against the model, 10x
phase space, generated and kept on the GPU), runs a quasi-Newton fit (the
library's projected limited-memory BFGS, at most 100 NLL + gradient
evaluations on the device) and ends with one exact Hessian.

* Admission by device memory: a job is admitted when a slot is free and its
  estimated resident bytes (event caches, from a per-model bytes-per-event
  figure measured on a small prototype) fit in the budget next to the jobs
  already running (the reference instead checks capacity once per analysis,
  DeviceManager.cu:223).
* Continuous batching: every admitted job runs in its own worker thread on
  its own CUDA stream, so jobs that arrive while others are on the GPU start
  as soon as a slot and memory free up, and their kernels overlap on the
  device; the C ABI calls release the GIL.
* Each job's fit loop runs in native code (``analysis.fit`` over
  ``ctpwa_fit``) with the GIL released: the four slots' evaluations do not
  queue behind one another's Python between device calls.
* Latency is recorded per evaluation and per fit; `summary()` reports
  p50/p99 and fits/hour.

Results do not depend on what else runs: every evaluation is deterministic
(fixed reduction order, no atomics) and private to its job's handle and
stream (tests/test_serving.py checks alone == in the mix).
"""
from __future__ import annotations

import math
import os
import queue
import shutil
import tempfile
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import workloads


@dataclass
class JobSpec:
    job_id: int
    model: str                 # workload template: "pipi_rho" or "pipi_3rho"
    n_data: int
    n_phsp: int
    seed: int
    arrival: float = 0.0       # seconds after the stream starts
    max_evals: int = 100
    precision: str = "mixed"
    # profile-likelihood scan after the fit: parameter `scan_param` fixed at
    # the fitted value + s * sigma for each s in scan_sigmas (sigma from the
    # job's Hessian), the other parameters refitted from the best fit
    scan_param: int = -1
    scan_sigmas: tuple = ()


@dataclass
class JobResult:
    job_id: int
    model: str
    n_data: int
    n_phsp: int
    precision: str
    nll: float = float("nan")
    params: Optional[np.ndarray] = None
    hessian: Optional[np.ndarray] = None
    n_evals: int = 0
    eval_ms: List[float] = field(default_factory=list)
    arrival: float = 0.0
    admitted: float = 0.0
    setup_done: float = 0.0
    finished: float = 0.0
    error: Optional[str] = None
    # phases of the service time (ms): toy-MC generation, handle creation
    # (model, kernels, angular pass), fit, Hessian, scan
    phase_ms: dict = field(default_factory=dict)
    # profile scan: (parameter value, NLL - best-fit NLL) per point
    scan: List[tuple] = field(default_factory=list)

    @property
    def fit_latency(self) -> float:
        return self.finished - self.arrival


def poisson_stream(rate: float, n_jobs: int, models=("pipi_rho", "pipi_3rho"), nd_range=(10_000, 2_000_000),
                   phsp_factor: int = 10, seed: int = 17, max_evals: int = 100, precision: str = "mixed"):
    """Seeded stream: exponential inter-arrival times at `rate` jobs/s, N_data
    log-uniform in nd_range, N_phsp = phsp_factor * N_data, models alternating."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    lo, hi = math.log(nd_range[0]), math.log(nd_range[1])
    for j in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        nd = int(round(math.exp(rng.uniform(lo, hi))))
        jobs.append(JobSpec(job_id=j, model=models[j % len(models)], n_data=nd, n_phsp=phsp_factor * nd,
                            seed=1000 + j, arrival=t, max_evals=max_evals, precision=precision))
    return jobs


class Server:
    """Runs fit jobs on one GPU with `slots` concurrent jobs and a device-memory budget."""

    def __init__(self, device: int = 0, slots: int = 4, budget_bytes: Optional[int] = None,
                 workdir: Optional[str] = None, batch: bool = False):
        import torch

        self.device = int(device)
        # batch=True: the fits' evaluations are gathered across the running
        # jobs into shared launches (one per model and precision and round)
        self.batch = None
        if batch:
            import ctpwa_b200

            self.batch = ctpwa_b200.EvalBatch(self.device)
        self.slots = int(slots)
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            budget_bytes = int(0.6 * free)
        self.budget = int(budget_bytes)
        base = workdir or ("/dev/shm" if os.path.isdir("/dev/shm") else None)
        self.workdir = tempfile.mkdtemp(prefix="ctpwa_serve_", dir=base)
        self._lock = threading.Lock()
        self._in_use = 0
        # one CUDA stream per slot, reused by the jobs that run in it and by
        # later servers of the process: the tensor allocator caches memory
        # per stream, so a new stream per job (or per server) would allocate
        # fresh device memory
        pool = Server._stream_pool.setdefault(self.device, [])
        while len(pool) < self.slots:
            pool.append(torch.cuda.Stream(device=self.device))
        self._streams: "queue.Queue" = queue.Queue()
        for st in pool[:self.slots]:
            self._streams.put(st)

    def close(self):
        shutil.rmtree(self.workdir, ignore_errors=True)
        if self.batch is not None:
            self.batch.close()
            self.batch = None

    # ----------------------------------------------------------- admission
    # resident device bytes per event of each model, shared by all servers of the process
    _bpe: dict = {}
    # the process's job streams per device
    _stream_pool: dict = {}

    def bytes_per_event(self, model: str) -> float:
        """Resident device bytes per event of a model, measured once per process on a prototype."""
        if model not in self._bpe:
            from . import analysis

            d = os.path.join(self.workdir, f"proto_{model}")
            cfg = workloads.make(model, d, n_phsp=20_000, n_data=2_000, n_bkg=0, accept_reject=False, seed=1,
                                 device=self.device)
            ana = analysis(cfg, device=self.device)
            self._bpe[model] = ana.deviceBytes() / float(sum(ana.getNEvents()))
            del ana
            shutil.rmtree(d, ignore_errors=True)
        return self._bpe[model]

    def job_bytes(self, spec: JobSpec) -> int:
        # resident caches plus, during set-up, the accept-reject candidates
        # (12x data: their momenta and the caches of the handle that weighs
        # them) and the transient momenta of the angular passes
        events = spec.n_data + spec.n_phsp
        cand = 12 * spec.n_data + 10_000
        return int(self.bytes_per_event(spec.model) * (events + cand) + 96 * (2 * events + 2 * cand))

    def try_reserve(self, nbytes: int) -> bool:
        with self._lock:
            if self._in_use + nbytes > self.budget:
                return False
            self._in_use += nbytes
            return True

    def release(self, nbytes: int):
        with self._lock:
            self._in_use -= nbytes

    # ----------------------------------------------------------- one job
    def run_job(self, spec: JobSpec, t0: float) -> JobResult:
        import torch

        from . import analysis

        res = JobResult(job_id=spec.job_id, model=spec.model, n_data=spec.n_data, n_phsp=spec.n_phsp,
                        precision=spec.precision, arrival=spec.arrival, admitted=time.perf_counter() - t0)
        d = os.path.join(self.workdir, f"job{spec.job_id}")
        stream = self._streams.get()
        try:
            with torch.cuda.device(self.device), torch.cuda.stream(stream):
                # toy-MC events generated and kept on the device, the job's
                # handle built from them (no file round trip)
                t1 = time.perf_counter()
                gen_ms = {}
                cfg, phsp, data = workloads.make_device(spec.model, d, spec.n_phsp, spec.n_data, seed=spec.seed,
                                                        device=self.device, timing=gen_ms)
                t2 = time.perf_counter()
                ana = analysis.from_device(cfg, phsp, data, device=self.device, precision=spec.precision)
                del phsp, data
                stream.synchronize()
                t3 = time.perf_counter()
                nV = ana.getNVector()
                truth = workloads.true_params(nV, ana.getFreeResParams()[0].numpy())
                rng = np.random.default_rng(spec.seed + 7)
                start = truth.copy()
                start[1:nV] *= 1.0 + 0.05 * rng.standard_normal(nV - 1)
                start[nV + 1:2 * nV] *= 1.0 + 0.05 * rng.standard_normal(nV - 1)
                start[2 * nV:] *= 1.0 + 0.002 * rng.standard_normal(start.size - 2 * nV)
                res.setup_done = time.perf_counter() - t0
                p, nll, n_evals, lat = self._fit(ana, start, spec, stream)
                stream.synchronize()
                t4 = time.perf_counter()
                H = ana.getHessian(p)
                stream.synchronize()
                t5 = time.perf_counter()
                res.phase_ms = {"generate": 1e3 * (t2 - t1), "handle": 1e3 * (t3 - t2), "fit": 1e3 * (t4 - t3),
                                "hessian": 1e3 * (t5 - t4)}
                if spec.scan_param >= 0 and spec.scan_sigmas:
                    res.scan = self._scan(ana, p, nll, H, spec, stream)
                    res.phase_ms["scan"] = 1e3 * (time.perf_counter() - t5)
                res.phase_ms.update({"generate." + k: v for k, v in gen_ms.items()})
                res.params = p.cpu().numpy()
                res.hessian = H.cpu().numpy()
                res.nll = nll
                res.n_evals = n_evals
                res.eval_ms = lat
                del ana
        except Exception as e:  # a failing job is reported, the server keeps going
            res.error = f"{type(e).__name__}: {e}"
        finally:
            stream.synchronize()
            self._streams.put(stream)
            shutil.rmtree(d, ignore_errors=True)
        res.finished = time.perf_counter() - t0
        return res

    def _fit(self, ana, start, spec: JobSpec, stream):
        """The library's fit driver (``analysis.fit``: projected limited-memory
        BFGS in native code, the GIL released, one host-buffer evaluation per
        function call on the job's stream); the first coupling stays at its
        start value (overall phase and scale of the couplings are not
        measured: example/fit.py:48 fixes it) and the resonance parameters
        within their bounds, as the reference's fit clamps them."""
        import torch

        # relative decrease at which the fit stops: in the mixed form the NLL
        # carries ~1e-4 to 1e-3 of rounding at these sizes, and a stop below it
        # turns into line searches that cannot find a decrease (49 evaluations
        # instead of 9 on a 2M-event job); 1e-10 of |NLL| is ~1e-4 at 1M
        # events, far below the 0.5 of one standard deviation
        ftol = 1e-10 if ana.getPrecision() == "mixed" else 1e-13
        x, nll, n_evals, _, _, lat = ana.fit(start, max_evals=spec.max_evals, history=20, ftol=ftol, gtol=1e-9,
                                             stream=stream, batch=self.batch)
        return torch.tensor(x, dtype=torch.float64, device=torch.device("cuda", self.device)), nll, n_evals, lat

    @staticmethod
    def _scan(ana, best, nll_best, H, spec: JobSpec, stream):
        """Profile-likelihood scan of parameter spec.scan_param around the
        fit: sigma from the inverse Hessian over the free parameters, one
        refit (parameter fixed) per point, started from the best fit."""
        import torch

        nV = ana.getNVector()
        n = best.numel()
        i = int(spec.scan_param)
        if not 0 <= i < n or i in (0, nV):
            raise ValueError(f"scan_param {i} is not a free parameter")
        free = np.ones(n, dtype=bool)
        free[0] = free[nV] = False
        # covariance on the device (FP64 inverse of the Hessian over the free parameters)
        sigma = float(torch.sqrt(ana.getCovariance(best, free=free, hessian=H)[i, i]))
        best = best.cpu().numpy()
        res = ana.getFreeResParams().numpy()
        lo = np.concatenate([np.full(2 * nV, -np.inf), res[1]])
        hi = np.concatenate([np.full(2 * nV, np.inf), res[2]])
        fr = free.astype(np.uint8)
        fr[i] = 0
        out = []
        for s_ in spec.scan_sigmas:
            x0 = best.copy()
            x0[i] = min(max(best[i] + float(s_) * sigma, lo[i]), hi[i])
            _, f, _, _, _, _ = ana.fit(x0, lower=lo, upper=hi, free=fr, max_evals=spec.max_evals, stream=stream)
            out.append((float(x0[i]), f - nll_best))
        return out

    # ----------------------------------------------------------- the stream
    def run(self, jobs: List[JobSpec], realtime: bool = True) -> List[JobResult]:
        """Serve `jobs` (arrival times in seconds from now when realtime)."""
        pending = sorted(jobs, key=lambda j: j.arrival)
        for j in pending:
            self.bytes_per_event(j.model)
        results = []
        done_q: "queue.Queue" = queue.Queue()
        running = {}
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=self.slots) as pool:
            while pending or running:
                now = time.perf_counter() - t0
                # admit arrived jobs in arrival order while slots and memory allow
                while pending and len(running) < self.slots and (not realtime or pending[0].arrival <= now):
                    spec = pending[0]
                    nb = self.job_bytes(spec)
                    if nb > self.budget:
                        pending.pop(0)
                        r = JobResult(job_id=spec.job_id, model=spec.model, n_data=spec.n_data,
                                      n_phsp=spec.n_phsp, precision=spec.precision, arrival=spec.arrival,
                                      finished=now, error=f"needs {nb} bytes, budget {self.budget}")
                        results.append(r)
                        continue
                    if not self.try_reserve(nb):
                        break
                    pending.pop(0)
                    if not realtime:
                        spec.arrival = now
                    fut = pool.submit(self.run_job, spec, t0)
                    running[spec.job_id] = nb
                    fut.add_done_callback(lambda f, jid=spec.job_id: done_q.put((jid, f)))
                # wait for a completion or the next arrival
                timeout = 0.05
                if pending and realtime and len(running) < self.slots:
                    timeout = max(0.0, min(timeout, pending[0].arrival - (time.perf_counter() - t0)))
                try:
                    jid, f = done_q.get(timeout=timeout)
                except queue.Empty:
                    continue
                self.release(running.pop(jid))
                results.append(f.result())
        return sorted(results, key=lambda r: r.job_id)


def percentile(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else float("nan")


def summary(results: List[JobResult], wall_s: float) -> dict:
    ok = [r for r in results if r.error is None]
    evals = [x for r in ok for x in r.eval_ms]
    fits = [1e3 * r.fit_latency for r in ok]
    service = [1e3 * (r.finished - r.admitted) for r in ok]
    return {
        "jobs": len(results),
        "failed": len(results) - len(ok),
        "fits_per_hour": 3600.0 * len(ok) / wall_s if wall_s > 0 else float("nan"),
        "evals": len(evals),
        "eval_ms_p50": percentile(evals, 50),
        "eval_ms_p99": percentile(evals, 99),
        "fit_ms_p50": percentile(fits, 50),
        "fit_ms_p99": percentile(fits, 99),
        "service_ms_p50": percentile(service, 50),
        "service_ms_p99": percentile(service, 99),
        "phase_ms_p50": {k: percentile([r.phase_ms[k] for r in ok if k in r.phase_ms], 50)
                         for k in sorted({k for r in ok for k in r.phase_ms})},
        "slowest": _job_record(max(ok, key=lambda r: r.fit_latency)) if ok else None,
        "errors": [r.error for r in results if r.error][:5],
    }


def _job_record(r: JobResult) -> dict:
    """One job's size, evaluations and latency breakdown (ms): where a tail
    latency comes from."""
    return {"job": r.job_id, "model": r.model, "n_data": r.n_data, "n_phsp": r.n_phsp, "evals": r.n_evals,
            "fit_ms": 1e3 * r.fit_latency, "queue_ms": 1e3 * (r.admitted - r.arrival),
            "eval_ms_sum": float(np.sum(r.eval_ms)) if r.eval_ms else 0.0,
            "phase_ms": {k: round(v, 3) for k, v in r.phase_ms.items()}}


def main(argv=None):
    import argparse
    import json

    ap = argparse.ArgumentParser(description="Serve a Poisson stream of toy-MC fit jobs on one GPU")
    ap.add_argument("--rate", type=float, default=5.0)
    ap.add_argument("--jobs", type=int, default=20)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--nd-min", type=int, default=10_000)
    ap.add_argument("--nd-max", type=int, default=200_000)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--seed", type=int, default=17)
    ap.add_argument("--scan-param", type=int, default=-1,
                    help="after each fit, profile-scan this parameter index at +-1, +-2 sigma")
    a = ap.parse_args(argv)
    srv = Server(device=a.device, slots=a.slots)
    try:
        # untimed jobs of the largest size first: one-time process costs
        # (library and kernel loading, the per-model memory figure, growth of
        # the memory pools) are not stream latency
        srv.run([JobSpec(job_id=-1 - i, model=("pipi_rho", "pipi_3rho")[i % 2], n_data=a.nd_max, n_phsp=10 * a.nd_max,
                         seed=90 + i, max_evals=5, precision=a.precision) for i in range(a.slots)], realtime=False)
        jobs = poisson_stream(a.rate, a.jobs, nd_range=(a.nd_min, a.nd_max), precision=a.precision, seed=a.seed)
        if a.scan_param >= 0:
            for j in jobs:
                j.scan_param, j.scan_sigmas = a.scan_param, (-2.0, -1.0, 1.0, 2.0)
        t = time.perf_counter()
        res = srv.run(jobs)
        out = summary(res, time.perf_counter() - t)
        out.update({"rate_per_s": a.rate, "slots": a.slots, "precision": a.precision, "fit": "native projected L-BFGS"})
        print(json.dumps(out))
    finally:
        srv.close()


if __name__ == "__main__":
    main()
