"""Identical-particle symmetrisation (reference AmpCasDecay::buildPermTopologies,
src/AmpGen.cu:194-405): each chain with identical final-state particles is
summed over their permutations. Checked on the CPU oracle: the model lowering
adds one exchanged variant per chain, the intensity is invariant under the
exchange of the two identical particles, and the oracle's gradient agrees
with central finite differences."""
import numpy as np
import pytest

import ctpwa_b200
from ctpwa_b200 import workloads
from oracle.binding import Oracle


@pytest.fixture(scope="module")
def ksks(tmp_path_factory):
    d = tmp_path_factory.mktemp("ksks")
    cfg = workloads.make("ksks", d, n_phsp=3_000, n_data=700, n_bkg=0, accept_reject=False, seed=4,
                         gpu_generator=False)
    return d, cfg


def test_model_has_exchange_variants(ksks):
    _, cfg = ksks
    m = ctpwa_b200.describe(cfg)
    base = [g for g in m["groups"] if g["base"] < 0]
    var = [g for g in m["groups"] if g["base"] >= 0]
    assert len(base) == 2 and len(var) == 2
    for g in base:
        assert len(g["variants"]) == 1
        v = m["groups"][g["variants"][0]]
        assert v["sign"] == 1.0  # bosons
        # the variant reads the two K_S slots exchanged
        a, b = g["input_slot"], v["input_slot"]
        assert sorted(a) == sorted(b) and a != b
    # blocks live on base groups only
    assert all(m["groups"][b["group"]]["base"] < 0 for b in m["blocks"])


def test_intensity_invariant_under_exchange(ksks):
    d, cfg = ksks
    o = Oracle(cfg)
    p = workloads.true_params(o.nV, o.theta_init()[0])
    I1 = o.intensity(1, p)
    data = np.load(d / "data.npy")
    np.save(d / "data_swapped.npy", data[:, [1, 0, 2], :])
    text = open(cfg).read().replace(str(d / "data.npy"), str(d / "data_swapped.npy"))
    cfg2 = d / "swapped.yml"
    cfg2.write_text(text)
    I2 = Oracle(str(cfg2)).intensity(1, p)
    assert np.max(np.abs(I1 - I2) / np.abs(I1)) < 1e-12


def test_oracle_gradient_fd(ksks):
    _, cfg = ksks
    o = Oracle(cfg)
    p = workloads.true_params(o.nV, o.theta_init()[0])
    p[2 * o.nV:] *= 1.002
    _, g, _ = o.nll_grad(p)
    for j in range(p.size):
        h = 1e-6 * max(abs(p[j]), 1.0)
        q = p.copy()
        q[j] += h
        fp = o.nll_grad(q)[0]
        q[j] -= 2 * h
        fm = o.nll_grad(q)[0]
        assert abs((fp - fm) / (2 * h) - g[j]) <= 1e-6 * max(1.0, np.max(np.abs(g))), j
