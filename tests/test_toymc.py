import numpy as np

from ctpwa_b200 import toymc


def test_phase_space_kinematics():
    M, masses = 3.0969, (0.493677, 0.493677, 0.13495)
    p = toymc.phase_space(M, masses, 20000, 5)
    m2 = p[..., 0] ** 2 - np.sum(p[..., 1:] ** 2, axis=-1)
    assert np.allclose(np.sqrt(m2), np.array(masses)[None, :], rtol=1e-10)
    tot = p.sum(axis=1)
    assert np.allclose(tot[:, 0], M, rtol=1e-12) and np.allclose(tot[:, 1:], 0.0, atol=1e-12)


def test_phase_space_flat_dalitz():
    M, masses = 3.0969, (0.13975, 0.13975, 0.13495)
    p = toymc.phase_space(M, masses, 200000, 9)
    s12 = (p[:, 0] + p[:, 1])
    s12 = s12[:, 0] ** 2 - np.sum(s12[:, 1:] ** 2, axis=1)
    s13 = (p[:, 0] + p[:, 2])
    s13 = s13[:, 0] ** 2 - np.sum(s13[:, 1:] ** 2, axis=1)
    # flat Dalitz density: the mean of s13 at fixed s12 band is the band's midpoint
    lo, hi = 2.0, 2.5
    sel = (s12 > lo) & (s12 < hi)
    h, _ = np.histogram(s13[sel], bins=10)
    inner = h[2:-2]
    assert inner.std() / inner.mean() < 0.05


def test_deterministic_seed():
    a = toymc.phase_space(3.0969, (0.14, 0.14, 0.135), 100, 1)
    b = toymc.phase_space(3.0969, (0.14, 0.14, 0.135), 100, 1)
    assert np.array_equal(a, b)
