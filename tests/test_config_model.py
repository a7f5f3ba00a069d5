"""Config schema parsing and model lowering (host only), against expectations
derived by hand from the reference's rules (src/Config.cu, src/Info.cu,
src/AmpGen.cu:69-129 and :2009-2342, src/Analysis.cu:4382-4478)."""
import os
import warnings

import pytest

import ctpwa_b200
from ctpwa_b200 import workloads
from conftest import reference_root

HERE = os.path.dirname(os.path.abspath(__file__))


def _cfg(tmp_path, name):
    p = tmp_path / f"{name}.yml"
    p.write_text(workloads.config_text(name, "p.npy", "d.npy", "b.npy", 0.3))
    return str(p)


def test_pipi_rho_model(tmp_path):
    m = ctpwa_b200.describe(_cfg(tmp_path, "pipi_rho"))
    assert m["npol"] == 3  # J/psi (3) x three pions (1)
    assert m["amplitude_names"] == ["Jpsi→pi0+rho770_SL(3,1)_rho770→pip+pim_SL(1,1)"]
    assert m["param_names"] == [m["amplitude_names"][0], "rho770_mass", "rho770_width"]
    assert m["coupling"]["n_free"] == 1
    g = m["groups"][0]
    # J/psi(1-) -> rho(1-) pi0(0-): S=1 only, parity (-1)^L = -1 -> L = 1
    assert g["nodes"][0]["sls"] == [[3, 1]] and g["nodes"][1]["sls"] == [[1, 1]]
    s = m["slots"]
    assert [x["name"] for x in s] == ["rho770_mass", "rho770_width"]
    # default bounds: value +- 50 % of |value|
    assert s[0]["lower"] == pytest.approx(0.3875) and s[0]["upper"] == pytest.approx(1.1625)


def test_three_rho_shares_names(tmp_path):
    m = ctpwa_b200.describe(_cfg(tmp_path, "pipi_3rho"))
    assert len(m["amplitude_names"]) == 9
    assert m["coupling"]["n_free"] == 9
    assert [x["name"] for x in m["slots"]] == ["rho770_mass", "rho770_width", "rho1450_mass", "rho1450_width",
                                               "rho1700_mass", "rho1700_width"]
    # rho+ and rho- chains reuse the rho0 chain's theta slots
    th = [r["theta"] for b in m["blocks"] for r in b["res"]]
    assert th[:3] == th[3:6] == th[6:9] == [[0, 1], [2, 3], [4, 5]]


def test_kkpi_model(tmp_path):
    m = ctpwa_b200.describe(_cfg(tmp_path, "kkpi"))
    assert len(m["amplitude_names"]) == 7 and m["coupling"]["n_free"] == 7
    assert len(m["slots"]) == 9 and len(m["groups"]) == 5
    k2 = [g for g in m["groups"] if g["nodes"][0]["sls"] == [[5, 2]]]
    assert len(k2) == 2 and all(g["nodes"][1]["sls"] == [[1, 2]] for g in k2)  # D-wave barrier
    x = m["blocks"][-1]["res"][0]
    assert x["type"] == "Custom" and x["param_names"] == ["mass", "gKK", "gpipi"]


def test_feature_config(tmp_path):
    m = ctpwa_b200.describe(os.path.join(HERE, "golden", "features.yml"))
    names = m["amplitude_names"]
    # f0(980) 0+ is parity forbidden in J/psi -> eta f0: only the 1- group contributes for R_KK
    assert any("phi1020" in n for n in names) and not any("f0_980" in n for n in names)
    assert any("K1410" in n for n in names) and any("f2_1525" in n for n in names)
    # trans folds the R_Keta_1 chain onto R_Keta_0 with ratio -1: one fewer free coupling
    ratios = m["coupling"]["ratio"]
    assert sorted(set(ratios)) == [-1.0, 1.0]
    assert m["coupling"]["n_free"] == len(names) - ratios.count(-1.0)
    slots = {s["name"]: s for s in m["slots"]}
    assert slots["rho1700_width"]["lower"] == 0.2 and slots["rho1700_width"]["upper"] == 0.3
    assert slots["rho1700_mass"]["lower"] == 1.6 and slots["rho1700_mass"]["upper"] == 1.8
    assert "f2_1525_width" not in slots and "f2_1525_mass" in slots  # fix_var removes the slot
    assert "phi1020_mass" not in slots  # not free
    assert m["gauss"] and m["gauss"][0][2] == 0.01
    # K1410 in the folded chain shares the owner's theta slots
    k = [r["theta"] for b in m["blocks"] for r in b["res"] if r["name"] == "K1410"]
    assert len(k) == 2 and k[0] == k[1]


def test_invalid_config_is_not_valid(tmp_path):
    assert not ctpwa_b200.DecayInfo(str(tmp_path / "missing.yml")).isValid()
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        ana = ctpwa_b200.analysis(str(tmp_path / "missing.yml"))
    assert not ana.isValid() and any("not initialized" in str(x.message) for x in w)
    with pytest.raises(RuntimeError):
        ana.getNVector()


def test_bad_custom_expression_is_rejected(tmp_path):
    p = tmp_path / "bad.yml"
    p.write_text(workloads.config_text("kkpi", "p.npy", "d.npy").replace("Bf(1, q, q0, 3.0)", "Bf(L, q, q0, 3.0)"))
    with pytest.raises(RuntimeError, match="must be a number"):
        ctpwa_b200.describe(str(p))
    p.write_text(workloads.config_text("kkpi", "p.npy", "d.npy").replace("* Bf(", "* Foo("))
    with pytest.raises(RuntimeError, match="is not a function"):
        ctpwa_b200.describe(str(p))


def test_reference_example_config_parses():
    """The reference's own example config (flow maps, complex keys, Plot
    section) parses; it lists particles absent from Data.order, which the
    reference's reader rejects too."""
    root = reference_root()
    if root is None:
        pytest.skip("reference tree not present")
    ref = os.path.join(root, "example", "config.yml")
    with pytest.raises(RuntimeError, match="Data.order"):
        ctpwa_b200.describe(ref)


@pytest.mark.parametrize("expr,message", [
    ("BWR(mass, gKK, L)", "must be a number"),
    ("foo(m)", "is not a function"),
    ("2m", "malformed number"),
    ("1e", "exponent without digits"),
    ("mass +", "operand is expected"),
    ("(mass", "expected '\\)'"),
    ("exp m", "after a complete expression"),
    ("exp", "without an argument list"),
    ("BW(mass)", "BW takes"),
    ("Flatte(mass, gKK, 0.49)", "Flatte takes"),
    ("mass $ 2", "not part of the language"),
    ("mass * nope", "neither a parameter"),
])
def test_custom_expression_errors(tmp_path, expr, message):
    """Syntax and name errors of the custom-lineshape language are reported
    with the offending column, at model creation (no GPU needed)."""
    text = workloads.config_text("kkpi", "p.npy", "d.npy")
    old = 'expr: "Flatte(mass, gKK, gpipi, 0.493677, 0.493677, 0.13957, 0.13957) * Bf(1, q, q0, 3.0)"'
    assert old in text
    p = tmp_path / "bad.yml"
    p.write_text(text.replace(old, f'expr: "{expr}"'))
    with pytest.raises(RuntimeError, match=message):
        ctpwa_b200.describe(str(p))


@pytest.mark.parametrize("expr", ["-mass^2^0.5 + (m/gKK)^(1j*gKK) - -gpipi", "mass^-1^2 * 3*-m", ".5e+1*q0 + q0(m)",
                                  "BWR(mass, gKK) + BWR(mass, gKK, 2) + BWR(mass, gKK, 1, 5.0)"])
def test_custom_expression_accepted(tmp_path, expr):
    text = workloads.config_text("kkpi", "p.npy", "d.npy")
    old = 'expr: "Flatte(mass, gKK, gpipi, 0.493677, 0.493677, 0.13957, 0.13957) * Bf(1, q, q0, 3.0)"'
    p = tmp_path / "ok.yml"
    p.write_text(text.replace(old, f'expr: "{expr}"'))
    assert len(ctpwa_b200.describe(str(p))["param_names"]) > 0
