"""Benchmark / test workloads: the J/psi -> 3 meson models used to measure
this engine, as config.yml text plus seeded synthetic samples.

* ``pipi_rho``    J/psi -> pi+ pi- pi0, one chain rho(770) -> pi+ pi- (BWR, m and width free)
* ``pipi_3rho``   J/psi -> pi+ pi- pi0, chains rho0 pi0, rho+ pi-, rho- pi+, each with
                  rho(770), rho(1450), rho(1700) (BWR; masses/widths free, shared by name)
* ``kkpi``        J/psi -> K+ K- pi0: K*(892)+-, K*(1410)+- (J=1), K*2(1430)+- (J=2, D wave)
                  as BWR plus a K+K- J=1 state with a custom Flatte lineshape
                  (mass 1.68, couplings 0.3 / 0.1 to KK / pipi); all parameters free

Samples are uniform three-body phase space (seeded) for phsp and background;
data are drawn by accept-reject against the model at the true couplings
(|v| in [0.1, 1], uniform phase, first coupling 1 + 0i, seeded) using the
engine's per-event intensities, or taken as flat phase space when
``accept_reject=False`` (enough for parity checks). With a background sample
of weight w, the data hold background events too (n_data in all, the rest
drawn against the model), per ``data_bkg``:

* ``"draw"`` (default): round(w n_bkg) events of the background's
  distribution (uniform phase space, their own seed), the background that
  the subtraction removes. Without them the subtracted density is negative
  wherever the model is small, and the likelihood falls by thousands of units
  from the generating parameters.
* ``"sample"``: the background sample's own n_bkg events. Every subtracted
  event then enters the NLL with net weight 1 - w > 0, so the likelihood is
  bounded below. With independent background events it is not: each
  subtracted event contributes +w log f at its own position, and an
  amplitude zero placed on it sends the NLL to -infinity (for the three-chain
  rho model such wells lie a few tens of NLL units below the generating
  point).
* ``"none"``: signal events only.
"""
from __future__ import annotations

import math
import os
from pathlib import Path

import numpy as np

from . import toymc

M_JPSI = 3.0969
M_PIC = 0.13975
M_PI0 = 0.13495
M_K = 0.493677

_PARTICLES_PIPI = """Particles:
  Jpsi: {J: 1, P: -1, mass: 3.0969}
  pip:  {J: 0, P: -1, mass: 0.13975}
  pim:  {J: 0, P: -1, mass: 0.13975}
  pi0:  {J: 0, P: -1, mass: 0.13495}
"""

_TEMPLATES = {
    "pipi_rho": _PARTICLES_PIPI + """Data:
  order: [pip, pim, pi0]
  data: [npy, "@DATA@"]
  phsp: [npy, "@PHSP@"]
@BKG@DecayChains:
  rho:
    Jpsi: [[pi0, R_pm]]
    R_pm: [pip, pim]
    intermediates:
      R_pm:
        - [J: 1, P: -1]: [rho770]
Resonances:
  rho770: {J: 1, P: -1, model: BWR, parameters: [0.775, 0.149], free: [0, 1]}
""",
    "pipi_3rho": _PARTICLES_PIPI + """Data:
  order: [pip, pim, pi0]
  data: [npy, "@DATA@"]
  phsp: [npy, "@PHSP@"]
@BKG@DecayChains:
  rho0:
    Jpsi: [[pi0, R_pm]]
    R_pm: [pip, pim]
    intermediates:
      R_pm:
        - [J: 1, P: -1]: [rho770, rho1450, rho1700]
  rhop:
    Jpsi: [[pim, R_p0]]
    R_p0: [pip, pi0]
    intermediates:
      R_p0:
        - [J: 1, P: -1]: [rho770, rho1450, rho1700]
  rhom:
    Jpsi: [[pip, R_m0]]
    R_m0: [pim, pi0]
    intermediates:
      R_m0:
        - [J: 1, P: -1]: [rho770, rho1450, rho1700]
Resonances:
  rho770:  {J: 1, P: -1, model: BWR, parameters: [0.775, 0.149], free: [0, 1]}
  rho1450: {J: 1, P: -1, model: BWR, parameters: [1.465, 0.400], free: [0, 1]}
  rho1700: {J: 1, P: -1, model: BWR, parameters: [1.720, 0.250], free: [0, 1]}
""",
    "kkpi": """Particles:
  Jpsi: {J: 1, P: -1, mass: 3.0969}
  Kp:   {J: 0, P: -1, mass: 0.493677}
  Km:   {J: 0, P: -1, mass: 0.493677}
  pi0:  {J: 0, P: -1, mass: 0.13495}
Data:
  order: [Kp, Km, pi0]
  data: [npy, "@DATA@"]
  phsp: [npy, "@PHSP@"]
@BKG@DecayChains:
  kstp:
    Jpsi: [[Km, R_Kp]]
    R_Kp: [Kp, pi0]
    intermediates:
      R_Kp:
        - [J: 1, P: -1]: [Kst892, Kst1410]
        - [J: 2, P: +1]: [Kst2_1430]
  kstm:
    Jpsi: [[Kp, R_Km]]
    R_Km: [Km, pi0]
    intermediates:
      R_Km:
        - [J: 1, P: -1]: [Kst892, Kst1410]
        - [J: 2, P: +1]: [Kst2_1430]
  xkk:
    Jpsi: [[pi0, R_KK]]
    R_KK: [Kp, Km]
    intermediates:
      R_KK:
        - [J: 1, P: -1]: [X1680]
Resonances:
  Kst892:    {J: 1, P: -1, model: BWR, parameters: [0.8955, 0.047], free: [0, 1]}
  Kst1410:   {J: 1, P: -1, model: BWR, parameters: [1.414, 0.232], free: [0, 1]}
  Kst2_1430: {J: 2, P: 1, model: BWR, parameters: [1.4256, 0.0985], free: [0, 1]}
  X1680:
    J: 1
    P: -1
    model: Custom
    paramValues: [1.68, 0.3, 0.1]
    paramNames: [mass, gKK, gpipi]
    free: [0, 1, 2]
    expr: "Flatte(mass, gKK, gpipi, 0.493677, 0.493677, 0.13957, 0.13957) * Bf(1, q, q0, 3.0)"
""",
    # identical final-state particles (K_S K_S): every chain is summed over the
    # exchange of the two K_S (Constraints.identical)
    "ksks": """Particles:
  Jpsi: {J: 1, P: -1, mass: 3.0969}
  Ks1:  {J: 0, P: -1, mass: 0.497611}
  Ks2:  {J: 0, P: -1, mass: 0.497611}
  pi0:  {J: 0, P: -1, mass: 0.13495}
Data:
  order: [Ks1, Ks2, pi0]
  data: [npy, "@DATA@"]
  phsp: [npy, "@PHSP@"]
@BKG@DecayChains:
  kst:
    Jpsi: [[Ks2, R_K]]
    R_K: [Ks1, pi0]
    intermediates:
      R_K:
        - [J: 1, P: -1]: [Kst892]
  f2:
    Jpsi: [[pi0, R_KK]]
    R_KK: [Ks1, Ks2]
    intermediates:
      R_KK:
        - [J: 2, P: 1]: [f2_1525]
Resonances:
  Kst892:  {J: 1, P: -1, model: BWR, parameters: [0.8955, 0.047], free: [0, 1]}
  f2_1525: {J: 2, P: 1, model: BWR, parameters: [1.5174, 0.086], free: [0, 1]}
Constraints:
  identical: [[Ks1, Ks2]]
""",
}
MASSES = {
    "pipi_rho": (M_PIC, M_PIC, M_PI0),
    "pipi_3rho": (M_PIC, M_PIC, M_PI0),
    "kkpi": (M_K, M_K, M_PI0),
    "ksks": (0.497611, 0.497611, M_PI0),
}

# sizes (phsp, data, bkg, bkg weight) of the measured configurations
SIZES = {
    "pipi_rho": (200_000, 20_000, 0, None),
    "pipi_3rho": (5_000_000, 500_000, 50_000, 0.8),
    "kkpi": (10_000_000, 1_000_000, 100_000, 0.3),
    "ksks": (1_000_000, 100_000, 0, None),
}


def config_text(name, phsp, data, bkg=None, bkg_weight=None):
    bkg_block = ""
    if bkg is not None:
        bkg_block = f'  bkg: [npy, "{bkg}"]\n'
        if bkg_weight is not None:
            bkg_block += f"  bkg_weights: [{bkg_weight}]\n"
    return _TEMPLATES[name].replace("@PHSP@", str(phsp)).replace("@DATA@", str(data)).replace("@BKG@", bkg_block)


def true_params(n_vector, theta_init, seed=4001):
    """Seeded couplings |v| ~ U[0.1, 1], phase ~ U[0, 2pi), first = 1 + 0i; theta at its initial values."""
    rng = np.random.default_rng(seed)
    mag = rng.uniform(0.1, 1.0, n_vector)
    ph = rng.uniform(0.0, 2.0 * math.pi, n_vector)
    re, im = mag * np.cos(ph), mag * np.sin(ph)
    re[0], im[0] = 1.0, 0.0
    return np.concatenate([re, im, np.asarray(theta_init, dtype=np.float64)])


def params_for(model):
    """True parameters of a lowered model (``describe``): seeded couplings and initial theta."""
    return true_params(int(model["coupling"]["n_free"]), [s["init"] for s in model["slots"]])


def _gen(M, masses, n, seed, gpu, device):
    if gpu and n >= 200_000:
        return toymc.phase_space_gpu(M, masses, n, seed, device=f"cuda:{device}")
    return toymc.phase_space(M, masses, n, seed)


def make(name, outdir, n_phsp=None, n_data=None, n_bkg=None, bkg_weight=None, seed=0, accept_reject=True,
         device=0, gpu_generator=None, intensity=None, params_fn=None, data_bkg="draw"):
    """Write samples + config.yml for workload `name` into outdir; returns the config path.

    accept_reject=True draws the data sample against the model at the true
    parameters; otherwise data are flat phase space. The per-candidate
    intensities come from ``intensity(config_path, params)`` (intensities of
    the config's data sample) when given, else from the GPU engine. Large
    samples are generated on the GPU when one is present (gpu_generator=None)
    or when gpu_generator=True."""
    sp, sd, sb, sw = SIZES[name]
    n_phsp = sp if n_phsp is None else n_phsp
    n_data = sd if n_data is None else n_data
    n_bkg = sb if n_bkg is None else n_bkg
    bkg_weight = sw if bkg_weight is None else bkg_weight
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    masses = MASSES[name]
    if gpu_generator is None:
        try:
            import torch

            gpu_generator = torch.cuda.is_available()
        except Exception:
            gpu_generator = False
    phsp = _gen(M_JPSI, masses, n_phsp, 1001 + seed, gpu_generator, device)
    toymc.write_npy(out / "phsp.npy", phsp)
    bkg_path, bkg = None, None
    if n_bkg:
        bkg = _gen(M_JPSI, masses, n_bkg, 3001 + seed, gpu_generator, device)
        toymc.write_npy(out / "bkg.npy", bkg)
        bkg_path = str(out / "bkg.npy")
    if accept_reject:
        n_in = bkg_in_data(n_data, n_bkg, bkg_weight, data_bkg)
        data = _accept_reject(name, out, masses, n_data - n_in, seed, device, gpu_generator, intensity, params_fn)
        if n_in and data_bkg == "sample":
            data = np.concatenate([data, bkg[:n_in]])
        elif n_in:
            data = np.concatenate([data, _gen(M_JPSI, masses, n_in, 4001 + seed, gpu_generator, device)])
    else:
        data = _gen(M_JPSI, masses, n_data, 2001 + seed, gpu_generator, device)
    toymc.write_npy(out / "data.npy", data)
    cfg = out / "config.yml"
    cfg.write_text(config_text(name, str(out / "phsp.npy"), str(out / "data.npy"), bkg_path, bkg_weight))
    return str(cfg)


def bkg_in_data(n_data, n_bkg, bkg_weight, data_bkg="draw"):
    """Background events in a data sample of n_data whose background sample
    (n_bkg events of weight bkg_weight) is subtracted: round(w n_bkg) for
    data_bkg "draw", n_bkg for "sample", 0 for "none"; at most n_data."""
    if data_bkg not in ("draw", "sample", "none"):
        raise ValueError("data_bkg must be 'draw', 'sample' or 'none'")
    if not n_bkg or not bkg_weight or bkg_weight <= 0 or data_bkg == "none":
        return 0
    n = int(n_bkg) if data_bkg == "sample" else int(round(float(bkg_weight) * int(n_bkg)))
    return min(int(n_data), n)


def _gpu_intensity(device):
    def run(cfg, params):
        import torch

        from . import analysis

        ana = analysis(str(cfg), device=device)
        p = torch.tensor(params, dtype=torch.float64, device=f"cuda:{device}")
        I = ana.getIntensity(p, kind=1).cpu().numpy()
        del ana
        return I

    return run


def _accept_reject(name, out, masses, n_data, seed, device, gpu_generator, intensity=None, params_fn=None):
    if intensity is None:
        intensity = _gpu_intensity(device)
    ncand = int(n_data * 12) + 10_000
    cand = _gen(M_JPSI, masses, ncand, 5001 + seed, gpu_generator, device)
    toymc.write_npy(out / "cand.npy", cand)
    tiny = toymc.phase_space(M_JPSI, masses, 1000, 7001 + seed)
    toymc.write_npy(out / "tiny.npy", tiny)
    cfg = out / "cand.yml"
    cfg.write_text(config_text(name, str(out / "tiny.npy"), str(out / "cand.npy")))
    if params_fn is None:
        from . import describe

        p = params_for(describe(str(cfg)))
    else:
        p = params_fn(str(cfg))
    I = intensity(cfg, p)
    sel = toymc.accept_reject(cand, I, seed=6001 + seed, safety=1.2)
    while sel.shape[0] < n_data:  # rare: top up from a fresh candidate batch
        more = _gen(M_JPSI, masses, ncand, 8001 + seed + sel.shape[0], gpu_generator, device)
        toymc.write_npy(out / "cand.npy", more)
        I2 = intensity(cfg, p)
        sel = np.concatenate([sel, toymc.accept_reject(more, I2, seed=9001 + seed, safety=1.2)])
    for f in ("cand.npy", "tiny.npy", "cand.yml"):
        try:
            os.remove(out / f)
        except OSError:
            pass
    return sel[:n_data]


def make_device_samples(name, outdir, n_phsp, n_data, n_bkg=0, bkg_weight=None, seed=0, device=0, data_bkg="draw"):
    """Workload `name` generated and kept on the GPU, background included
    (in the data too, see the module docstring): returns (config_path, phsp,
    data, bkg, weights) for
    ``analysis.from_device(config_path, phsp, data, bkg, weights=weights)``
    (bkg None when n_bkg is 0; weights: None or [None, None, bkg weights])."""
    import torch

    w = SIZES[name][3] if bkg_weight is None else bkg_weight
    n_in = bkg_in_data(n_data, n_bkg, w, data_bkg)
    cfg, phsp, data = make_device(name, outdir, n_phsp, n_data - n_in, seed=seed, device=device)
    if not n_bkg:
        return cfg, phsp, data, None, None
    bkg = toymc.phase_space_device(M_JPSI, MASSES[name], n_bkg, 3001 + seed, device=device)
    if n_in and data_bkg == "sample":
        data = torch.cat([data, bkg[:n_in]])
    elif n_in:
        data = torch.cat([data, toymc.phase_space_device(M_JPSI, MASSES[name], n_in, 4001 + seed, device=device)])
    wt = torch.full((n_bkg,), float(w), dtype=torch.float64, device=bkg.device)
    return cfg, phsp, data, bkg, [None, None, wt]


def make_device(name, outdir, n_phsp, n_data, seed=0, device=0, safety=1.2, timing=None):
    """Toy-MC samples of workload `name` generated and kept on the GPU:
    phase space from the seeded GPU generator, data by accept-reject of GPU
    candidates against the model's intensity at the true parameters (the
    candidates' intensities from an in-memory analysis, the draw on the
    device). Writes only config.yml (its Data entries name no files that are
    read) and returns (config_path, phsp, data) with float64 CUDA tensors
    [n, 3, 4] for ``analysis.from_device``. `timing` (a dict) receives the
    host time of each step in ms."""
    import time

    import torch

    from . import analysis, describe

    clock = [time.perf_counter()]

    def lap(key):
        if timing is not None:
            torch.cuda.current_stream(device).synchronize()
            t = time.perf_counter()
            timing[key] = timing.get(key, 0.0) + 1e3 * (t - clock[0])
            clock[0] = t

    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    masses = MASSES[name]
    dev = f"cuda:{device}"
    cfg = out / "config.yml"
    cfg.write_text(config_text(name, "in-memory-phsp", "in-memory-data"))
    phsp = toymc.phase_space_device(M_JPSI, masses, n_phsp, 1001 + seed, device=device)
    tiny = toymc.phase_space_device(M_JPSI, masses, 1000, 7001 + seed, device=device)
    p = torch.tensor(params_for(describe(str(cfg))), dtype=torch.float64, device=dev)
    lap("phsp")
    gen = torch.Generator(device=dev)
    gen.manual_seed(6001 + seed)
    # The first batch has 12 candidates per event; each later one is sized
    # from the acceptance measured so far (15 % margin) but holds no more
    # candidates than the first, so the device memory a caller reserves for
    # the first batch bounds every batch. (A fixed 12x per missing event
    # took ~15 batches, each with its own handle, on a model accepting 1/28.)
    chunks, have, batch, tried = [], 0, 0, 0
    cap = int(n_data * 12) + 10_000
    while have < n_data:
        if batch == 0:
            ncand = cap
        else:
            acc = max(have, 1) / tried
            ncand = min(cap, int(1.15 * (n_data - have) / acc) + 10_000)
        cand = toymc.phase_space_device(M_JPSI, masses, ncand, 5001 + seed + 7919 * batch, device=device)
        lap("candidates")
        ana = analysis.from_device(str(cfg), tiny, cand, device=device, fp64_only=True)
        lap("cand_handle")
        I = ana.getIntensity(p, kind=1)
        del ana
        u = torch.rand(ncand, generator=gen, dtype=torch.float64, device=dev) * (safety * I.max())
        sel = cand[u < I]
        lap("select")
        chunks.append(sel)
        have += sel.shape[0]
        tried += ncand
        batch += 1
    data = torch.cat(chunks)[:n_data].contiguous()
    return str(cfg), phsp, data
