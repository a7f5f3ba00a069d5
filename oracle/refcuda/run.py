"""Child process driving the reference CUDA build — test infrastructure.

python -m oracle.refcuda.run {f64|f32} job.json out.npz

job.json: {"config": path, "params": [[...], ...], "hessian": bool,
"timing": n}. Calls only the reference's public API (ctpwa.analysis,
getNLL + torch.autograd.grad, getHessian, the layout queries), the way
example/fit.py does.
"""
import json
import sys
import time

import numpy as np


def main():
    prec, job_path, out_path = sys.argv[1], sys.argv[2], sys.argv[3]
    job = json.load(open(job_path))
    import torch  # the extension links torch's libraries

    from oracle.refcuda import library

    sys.path.insert(0, str(library(prec).parent))
    import ctpwa  # noqa: E402  (the reference's own module)

    t0 = time.perf_counter()
    ana = ctpwa.analysis(job["config"])
    torch.cuda.synchronize()
    init_s = time.perf_counter() - t0
    if not ana.isValid():
        raise SystemExit("reference analysis is not valid for " + job["config"])
    meta = {
        "nV": int(ana.getNVector()),
        "nT": int(ana.getNFreeTheta()),
        "nP": int(ana.getNParams()),
        "names": list(ana.getParamNames()),
        "amplitude_names": [str(x) for x in ana.getAmplitudeNames()],
        "npol": int(ana.getNPolarizations()),
        "init_s": init_s,
    }
    out = {"free_res_params": np.asarray(ana.getFreeResParams().cpu().numpy(), dtype=np.float64)}
    nll, grad, hess = [], [], []
    for p in job["params"]:
        pt = torch.tensor(p, dtype=torch.float64, device="cuda", requires_grad=True)
        v = ana.getNLL(pt)
        (g,) = torch.autograd.grad(v, pt)
        nll.append(float(v.detach()))
        grad.append(g.detach().cpu().numpy())
        if job.get("hessian"):
            hess.append(ana.getHessian(pt.detach()).cpu().numpy())
    out["nll"] = np.array(nll)
    out["grad"] = np.array(grad) if grad else np.zeros((0, meta["nP"]))
    if hess:
        out["hessian"] = np.array(hess)
    n = int(job.get("timing") or 0)
    if n and job["params"]:
        base = np.array(job["params"][0], dtype=np.float64)
        nV, nT = meta["nV"], meta["nT"]
        rng = np.random.default_rng(123)
        times = []
        for i in range(n + 3):
            q = base.copy()
            q[2 * nV:] *= 1 + 1e-4 * rng.standard_normal(nT)  # resonance parameters move every evaluation
            pt = torch.tensor(q, dtype=torch.float64, device="cuda", requires_grad=True)
            torch.cuda.synchronize()
            t = time.perf_counter()
            v = ana.getNLL(pt)
            (g,) = torch.autograd.grad(v, pt)
            torch.cuda.synchronize()
            if i >= 3:
                times.append(time.perf_counter() - t)
        out["eval_s"] = np.array(times)
        if job.get("hessian"):
            pt = torch.tensor(base, dtype=torch.float64, device="cuda")
            ts = []
            for i in range(3):
                torch.cuda.synchronize()
                t = time.perf_counter()
                ana.getHessian(pt)
                torch.cuda.synchronize()
                ts.append(time.perf_counter() - t)
            out["hessian_s"] = np.array(ts)
    out["meta"] = np.array(json.dumps(meta))
    np.savez(out_path, **out)


if __name__ == "__main__":
    main()
