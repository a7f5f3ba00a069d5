"""Reference CUDA build as a second oracle — test infrastructure, not product code.

The reference's own `ctpwa` extension, built from its sources by
oracle/refcuda/build.py into oracle/_ref/cuda_{f64,f32}/ctpwa.so, is driven
in a child process (oracle/refcuda/run.py): the two precisions are the same
module name, and a failure of the reference stays out of the test process.

The reference reads samples from `.dat` text files (E px py pz per line, one
line per final-state particle in Data.order; src/Analysis.cu:58-176) and its
YAML through the stand-in yaml-cpp (which reads a PyYAML node tree written
beside the config). `dat_config` rewrites a workload config (npy samples) to
that form; the product reads the same `.dat` files, so both see identical
inputs.
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
BUILD = ROOT / "oracle" / "_ref"


def library(precision: str) -> Path:
    return BUILD / f"cuda_{precision}" / "ctpwa.so"


def available(precision: str = "f64") -> bool:
    return library(precision).exists()


def write_dat(npy_path, dat_path):
    """Sample (N, n_final, 4) float64 .npy -> .dat text, 17 significant digits
    (exact round trip through the reference's istream >> double)."""
    a = np.load(npy_path)
    with open(dat_path, "w") as f:
        np.savetxt(f, a.reshape(-1, 4), fmt="%.17g")


def dat_config(cfg_path, out_dir=None) -> str:
    """Copy of a config whose npy samples are replaced by .dat files (written
    beside it) and whose PyYAML node tree is written for the stand-in yaml-cpp.
    Returns the new config path."""
    from .yaml_nodes import write_nodes

    cfg_path = Path(cfg_path)
    out = Path(out_dir) if out_dir else cfg_path.parent
    out.mkdir(parents=True, exist_ok=True)
    text = cfg_path.read_text()

    def repl(m):
        src = Path(m.group(2))
        if not src.is_absolute():
            src = cfg_path.parent / src
        dat = out / (src.stem + ".dat")
        if not dat.exists():
            write_dat(src, dat)
        return f'{m.group(1)}[dat, "{dat}"]'

    text = re.sub(r'(\b(?:data|phsp|bkg|phsp_truth):\s*)\[npy,\s*"([^"]+)"\]', repl, text)
    new = out / (cfg_path.stem + "_dat.yml")
    new.write_text(text)
    write_nodes(new)
    return str(new)


def run(precision: str, cfg: str, params=(), hessian=False, timing=0, timeout=1800):
    """Evaluate the reference build on `cfg` (a dat_config output) in a child
    process. Returns a dict: layout (nV, nT, names, free_res_params,
    amplitude_names, npol), and per params vector: nll, grad, hessian (when
    asked), plus timing: seconds per getNLL + autograd evaluation over
    `timing` evaluations with the resonance parameters perturbed."""
    import tempfile

    with tempfile.TemporaryDirectory(prefix="ctpwa_refrun_") as d:
        job = Path(d) / "job.json"
        outp = Path(d) / "out.npz"
        job.write_text(json.dumps({"config": str(cfg), "params": [list(map(float, p)) for p in params],
                                   "hessian": bool(hessian), "timing": int(timing)}))
        env = dict(os.environ)
        env["PYTHONPATH"] = str(ROOT) + os.pathsep + env.get("PYTHONPATH", "")
        r = subprocess.run([sys.executable, "-m", "oracle.refcuda.run", precision, str(job), str(outp)],
                           capture_output=True, text=True, timeout=timeout, env=env, cwd=str(Path(cfg).parent))
        if r.returncode != 0 or not outp.exists():
            tail = (r.stdout[-3000:] + "\n" + r.stderr[-3000:]).strip()
            raise RuntimeError(f"reference build run failed (rc {r.returncode}):\n{tail}")
        z = np.load(outp, allow_pickle=False)
        res = {k: z[k] for k in z.files}
        meta = json.loads(str(res.pop("meta")))
        res.update(meta)
        res["log"] = r.stdout[-20000:]
        return res
