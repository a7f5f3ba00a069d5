"""The library's model lowering against an independent restatement
(oracle/lowering.py: PyYAML and the LS-coupling rules, no C++ front end):
amplitude names and order, free resonance parameters with their values and
bounds, and the number of free couplings, on the workload configurations and
on variants that reach more of the rules (several waves at one vertex, a
fixed resonance, `free: [-1]`, `free_range`)."""
import numpy as np
import pytest

import ctpwa_b200
from ctpwa_b200 import workloads
from oracle import lowering


def _check(cfg):
    d = ctpwa_b200.describe(str(cfg))
    r = lowering.lower(str(cfg))
    assert r["amplitude_names"] == d["amplitude_names"]
    assert [s[0] for s in r["slots"]] == [s["name"] for s in d["slots"]]
    for (_, v, lo, hi), s in zip(r["slots"], d["slots"]):
        np.testing.assert_allclose([v, lo, hi], [s["init"], s["lower"], s["upper"]], rtol=1e-12)
    assert r["n_free"] == d["coupling"]["n_free"]
    assert d["param_names"] == r["amplitude_names"] + [s[0] for s in r["slots"]]
    assert (r["npol"], r["npol_total"]) == (d["npol"], d["npol_total"])
    # the library lists the kept polarisations only when some are dropped
    assert r["pol_map"] == (list(d["pol_map"]) or list(range(d["npol_total"])))
    return r


@pytest.mark.parametrize("name", ["pipi_rho", "pipi_3rho", "kkpi", "ksks"])
def test_workload_lowering_matches_restatement(tmp_path, name):
    p = tmp_path / "c.yml"
    p.write_text(workloads.config_text(name, "p.npy", "d.npy"))
    _check(p)


def test_lowering_variants_match_restatement(tmp_path):
    base = workloads.config_text("pipi_3rho", "p.npy", "d.npy")
    # a resonance with every parameter free, one with explicit ranges, one fixed
    text = base.replace("rho770:  {J: 1, P: -1, model: BWR, parameters: [0.775, 0.149], free: [0, 1]}",
                        "rho770:  {J: 1, P: -1, model: BWR, parameters: [0.775, 0.149], free: [-1]}")
    text = text.replace("rho1450: {J: 1, P: -1, model: BWR, parameters: [1.465, 0.400], free: [0, 1]}",
                        "rho1450: {J: 1, P: -1, model: BWR, parameters: [1.465, 0.400], free: [1], "
                        "free_range: [[0.3, 0.5]]}")
    text = text.replace("rho1700: {J: 1, P: -1, model: BWR, parameters: [1.720, 0.250], free: [0, 1]}",
                        "rho1700: {J: 1, P: -1, model: BWR, parameters: [1.720, 0.250]}")
    assert "free: [-1]" in text and "free_range" in text
    p = tmp_path / "v.yml"
    p.write_text(text)
    r = _check(p)
    assert [s[0] for s in r["slots"]] == ["rho770_mass", "rho770_width", "rho1450_width"]
    np.testing.assert_allclose(r["slots"][2][2:], [0.3, 0.5])


def test_polarisation_mask_and_shared_parameters_match_restatement(tmp_path):
    """The layout case of the reference-build comparison: J/psi with m = +-1
    only and a var_equal group tying K*(1410)'s width to K*(892)'s."""
    text = workloads.config_text("kkpi", "p.npy", "d.npy")
    text = text.replace("Jpsi: {J: 1, P: -1, mass: 3.0969}",
                        "Jpsi: {J: 1, P: -1, mass: 3.0969, polarization: [1, -1]}")
    text = text.replace("Resonances:", "Constraints:\n  var_equal:\n    - [Kst892_width, Kst1410_width]\nResonances:", 1)
    p = tmp_path / "m.yml"
    p.write_text(text)
    r = _check(p)
    assert r["npol"] == 2 and r["pol_map"] == [0, 2]
    assert "Kst1410_width" not in [s[0] for s in r["slots"]]


def test_vertices_with_several_waves_match_restatement(tmp_path):
    """A spin-1 bachelor: J/psi -> V f0 has the waves (3,0), (3,2) and
    J/psi -> V f2 five waves, each amplitude one product of the two vertices'
    waves, the top vertex's outermost."""
    p = tmp_path / "w.yml"
    p.write_text("""Particles:
  Jpsi: {J: 1, P: -1, mass: 3.0969}
  V:    {J: 1, P: -1, mass: 0.78265}
  pip:  {J: 0, P: -1, mass: 0.13957}
  pim:  {J: 0, P: -1, mass: 0.13957}
Data:
  order: [V, pip, pim]
  data: [npy, "d.npy"]
  phsp: [npy, "p.npy"]
DecayChains:
  pp:
    Jpsi: [[V, R_pp]]
    R_pp: [pip, pim]
    intermediates:
      R_pp:
        - [J: 0, P: 1]: [f0_980]
        - [J: 2, P: 1]: [f2_1270]
Resonances:
  f0_980:  {J: 0, P: 1, model: BWR, parameters: [0.990, 0.070], free: [0, 1]}
  f2_1270: {J: 2, P: 1, model: BWR, parameters: [1.2755, 0.1867], free: [0, 1]}
""")
    r = _check(p)
    assert r["amplitude_names"] == [
        "Jpsi→V+f0_980_SL(3,0)_f0_980→pip+pim_SL(1,0)",
        "Jpsi→V+f0_980_SL(3,2)_f0_980→pip+pim_SL(1,0)",
        "Jpsi→V+f2_1270_SL(3,0)_f2_1270→pip+pim_SL(1,2)",
        "Jpsi→V+f2_1270_SL(3,2)_f2_1270→pip+pim_SL(1,2)",
        "Jpsi→V+f2_1270_SL(5,2)_f2_1270→pip+pim_SL(1,2)",
        "Jpsi→V+f2_1270_SL(7,2)_f2_1270→pip+pim_SL(1,2)",
        "Jpsi→V+f2_1270_SL(7,4)_f2_1270→pip+pim_SL(1,2)",
    ]


def test_ls_waves_rules():
    # J/psi (1-) -> pi0 (0-) + rho (1-): S = 1, L = 1 only
    assert lowering.ls_waves(1, -1, 0, -1, 1, -1) == [(3, 1)]
    # rho (1-) -> pi pi: P-wave
    assert lowering.ls_waves(1, -1, 0, -1, 0, -1) == [(1, 1)]
    # identical bosons: f2 (2+) -> KS KS allows L + S even only
    assert lowering.ls_waves(2, 1, 0, -1, 0, -1, identical=True) == [(1, 2)]
    assert lowering.ls_waves(1, -1, 0, -1, 0, -1, identical=True) == []
    # a baryonic vertex: 1/2+ -> 1/2+ 0-: S = 1/2, L = 1
    assert lowering.ls_waves(0.5, 1, 0.5, 1, 0, -1) == [(2, 1)]
