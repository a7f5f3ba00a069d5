"""CPU generation of a benchmark workload for the oracle — test infrastructure.

python -m oracle.cpu_workload OUTDIR [--name kkpi] [--seed S] [--fraction F] [--cand-factor C]

The same workload definition as the device benchmark (ctpwa_b200.workloads:
config text, seeded uniform three-body phase space for the phase-space and
background samples), generated on the host with numpy. The data sample is
left as C x n_data phase-space candidates (`data: cand.npy` in the config):
the caller opens the oracle on it, draws the data by accept-reject against
the model's oracle intensities and keeps the selected events in place
(Oracle.take), so every candidate's angular tensors are computed once. The
last n_bkg_in_data rows of cand.npy are the data's background events (kept
as they are, after the n_data - n_bkg_in_data accepted candidates).
params.json holds the true parameters (seeded couplings, initial resonance
parameters) and the data size to draw. Loads no product library: the
workload module is plain Python and the layout comes from the oracle.
"""
import argparse
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def generate(outdir, name="kkpi", seed=0, fraction=1.0, cand_factor=12):
    sys.path.insert(0, str(ROOT))
    from ctpwa_b200 import toymc, workloads  # plain Python: templates and the numpy generator

    from oracle.binding import Oracle

    n_p, n_d, n_b, w_b = workloads.SIZES[name]
    n_p, n_d, n_b = (max(100, int(round(x * fraction))) for x in (n_p, n_d, n_b))
    masses = workloads.MASSES[name]
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    toymc.write_npy(out / "phsp.npy", toymc.phase_space(workloads.M_JPSI, masses, n_p, 1001 + seed))
    bkg = None
    if n_b:
        toymc.write_npy(out / "bkg.npy", toymc.phase_space(workloads.M_JPSI, masses, n_b, 3001 + seed))
        bkg = str(out / "bkg.npy")
    # candidates for the signal part of the data, then the data's background
    # events (uniform phase space, as the device workload draws them)
    n_in = workloads.bkg_in_data(n_d, n_b, w_b)
    n_c = int(cand_factor * (n_d - n_in))
    cand = toymc.phase_space(workloads.M_JPSI, masses, n_c, 5001 + seed)
    if n_in:
        cand = np.concatenate([cand, toymc.phase_space(workloads.M_JPSI, masses, n_in, 4001 + seed)])
    toymc.write_npy(out / "cand.npy", cand)
    cfg = out / "config.yml"
    cfg.write_text(workloads.config_text(name, str(out / "phsp.npy"), str(out / "cand.npy"), bkg, w_b))
    # layout (number of couplings, initial resonance parameters) from the oracle on a tiny sample
    toymc.write_npy(out / "tiny.npy", toymc.phase_space(workloads.M_JPSI, masses, 200, 7001 + seed))
    tiny = out / "tiny.yml"
    tiny.write_text(workloads.config_text(name, str(out / "tiny.npy"), str(out / "tiny.npy")))
    o = Oracle(str(tiny))
    p = workloads.true_params(o.nV, o.theta_init()[0])
    nV, nT = o.nV, o.nT
    o.close()
    (out / "params.json").write_text(json.dumps({"true_params": [float(x) for x in p], "nV": nV, "nT": nT,
                                                 "n_data": n_d, "n_bkg_in_data": n_in, "sizes": [n_p, n_d, n_b],
                                                 "n_cand": n_c}))
    (out / "done").write_text("ok\n")
    return str(cfg)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("outdir")
    ap.add_argument("--name", default="kkpi")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--fraction", type=float, default=1.0)
    ap.add_argument("--cand-factor", type=float, default=12)
    a = ap.parse_args()
    print(generate(a.outdir, a.name, a.seed, a.fraction, a.cand_factor))
