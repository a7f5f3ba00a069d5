"""Seeded synthetic event samples for toy-MC fits and benchmarks.

* ``phase_space(M, masses, n, seed)`` draws events uniformly in three-body
  phase space (flat Dalitz density, isotropic orientation) by sequential
  two-body decays weighted by the product of breakup momenta and
  accept-reject on that weight.
* ``write_dat`` / ``write_npy`` store samples in the reference ``.dat`` text
  layout (one ``E px py pz`` line per final-state particle, in ``Data.order``)
  or as a float64 ``.npy`` array of shape ``(N, n_final, 4)``.
* ``accept_reject(p4, intensity, ...)`` keeps events with probability
  ``I / (safety * I_max)`` where the caller supplies per-event intensities.
"""
from __future__ import annotations

import numpy as np


def _breakup(m, m1, m2):
    q2 = (m * m - (m1 + m2) ** 2) * (m * m - (m1 - m2) ** 2)
    return np.sqrt(np.clip(q2, 0.0, None)) / (2.0 * m)


def _random_dir(rng, n):
    cth = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    sth = np.sqrt(1.0 - cth * cth)
    return np.stack([sth * np.cos(phi), sth * np.sin(phi), cth], axis=1)


def _boost(p4, beta):
    """Boost four-vectors p4 (n,4) by velocity beta (n,3) (active boost)."""
    b2 = np.sum(beta * beta, axis=1)
    gamma = 1.0 / np.sqrt(1.0 - b2)
    bp = np.sum(beta * p4[:, 1:], axis=1)
    coef = np.where(b2 > 0, (gamma - 1.0) / np.where(b2 > 0, b2, 1.0), 0.0)
    out = np.empty_like(p4)
    out[:, 0] = gamma * (p4[:, 0] + bp)
    out[:, 1:] = p4[:, 1:] + (coef * bp + gamma * p4[:, 0])[:, None] * beta
    return out


def phase_space(M, masses, n, seed):
    """Uniform three-body phase space for a parent of mass M at rest.

    Returns a float64 array (n, 3, 4) with (E, px, py, pz) per particle."""
    m1, m2, m3 = (float(x) for x in masses)
    rng = np.random.default_rng(seed)
    lo, hi = m1 + m2, M - m3
    # maximum of q(M; m12, m3) * q(m12; m1, m2) on a fine grid (x1.05 margin)
    grid = np.linspace(lo, hi, 20001)[1:-1]
    wmax = 1.05 * float(np.max(_breakup(M, grid, m3) * _breakup(grid, m1, m2)))
    out = np.empty((n, 3, 4))
    filled = 0
    while filled < n:
        k = max(4096, int((n - filled) * 2.2))
        m12 = rng.uniform(lo, hi, k)
        w = _breakup(M, m12, m3) * _breakup(m12, m1, m2)
        keep = rng.uniform(0.0, wmax, k) < w
        m12 = m12[keep]
        k = m12.size
        if k == 0:
            continue
        q3 = _breakup(M, m12, m3)
        d3 = _random_dir(rng, k)
        p3 = np.column_stack([np.sqrt(m3 * m3 + q3 * q3), -q3[:, None] * d3])
        e12 = np.sqrt(m12 * m12 + q3 * q3)
        q12 = _breakup(m12, m1, m2)
        d1 = _random_dir(rng, k)
        p1r = np.column_stack([np.sqrt(m1 * m1 + q12 * q12), q12[:, None] * d1])
        p2r = np.column_stack([np.sqrt(m2 * m2 + q12 * q12), -q12[:, None] * d1])
        beta = (q3[:, None] * d3) / e12[:, None]
        p1 = _boost(p1r, beta)
        p2 = _boost(p2r, beta)
        take = min(k, n - filled)
        out[filled:filled + take, 0] = p1[:take]
        out[filled:filled + take, 1] = p2[:take]
        out[filled:filled + take, 2] = p3[:take]
        filled += take
    return out


def phase_space_gpu(M, masses, n, seed, device="cuda", as_tensor=False):
    """Same generator on the GPU with torch's seeded Philox RNG (large samples).

    Returns a float64 numpy array (n, 3, 4), or the CUDA tensor (as_tensor)."""
    import torch

    m1, m2, m3 = (float(x) for x in masses)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    lo, hi = m1 + m2, M - m3
    grid = np.linspace(lo, hi, 20001)[1:-1]
    wmax = 1.05 * float(np.max(_breakup(M, grid, m3) * _breakup(grid, m1, m2)))
    f64 = dict(dtype=torch.float64, device=device)

    def brk(m, a, b):
        q2 = (m * m - (a + b) ** 2) * (m * m - (a - b) ** 2)
        return torch.sqrt(torch.clamp(q2, min=0.0)) / (2.0 * m)

    def rdir(k):
        cth = torch.rand(k, generator=gen, **f64) * 2.0 - 1.0
        phi = torch.rand(k, generator=gen, **f64) * (2.0 * np.pi)
        sth = torch.sqrt(1.0 - cth * cth)
        return torch.stack([sth * torch.cos(phi), sth * torch.sin(phi), cth], dim=1)

    out = torch.empty((n, 3, 4), **f64)
    filled = 0
    while filled < n:
        k = max(4096, int((n - filled) * 2.2))
        m12 = lo + (hi - lo) * torch.rand(k, generator=gen, **f64)
        w = brk(M, m12, m3) * brk(m12, m1, m2)
        keep = torch.rand(k, generator=gen, **f64) * wmax < w
        m12 = m12[keep]
        k = m12.numel()
        if k == 0:
            continue
        q3 = brk(M, m12, m3)
        d3 = rdir(k)
        p3 = torch.cat([torch.sqrt(m3 * m3 + q3 * q3)[:, None], -q3[:, None] * d3], dim=1)
        e12 = torch.sqrt(m12 * m12 + q3 * q3)
        q12 = brk(m12, m1, m2)
        d1 = rdir(k)
        p1r = torch.cat([torch.sqrt(m1 * m1 + q12 * q12)[:, None], q12[:, None] * d1], dim=1)
        p2r = torch.cat([torch.sqrt(m2 * m2 + q12 * q12)[:, None], -q12[:, None] * d1], dim=1)
        beta = (q3[:, None] * d3) / e12[:, None]
        b2 = (beta * beta).sum(1)
        gamma = 1.0 / torch.sqrt(1.0 - b2)
        coef = torch.where(b2 > 0, (gamma - 1.0) / torch.where(b2 > 0, b2, torch.ones_like(b2)), torch.zeros_like(b2))

        def boost(p):
            bp = (beta * p[:, 1:]).sum(1)
            return torch.cat([(gamma * (p[:, 0] + bp))[:, None],
                              p[:, 1:] + (coef * bp + gamma * p[:, 0])[:, None] * beta], dim=1)

        take = min(k, n - filled)
        out[filled:filled + take, 0] = boost(p1r)[:take]
        out[filled:filled + take, 1] = boost(p2r)[:take]
        out[filled:filled + take, 2] = p3[:take]
        filled += take
    return out if as_tensor else out.cpu().numpy()


def phase_space_device(M, masses, n, seed, device=0):
    """Uniform three-body phase space generated by the library's CUDA kernel
    (counter-based Philox random numbers: event i depends only on (seed, i)).

    Returns a float64 CUDA tensor (n, 3, 4) on `device`, written on its
    current stream."""
    import ctypes

    import torch

    from . import _lib

    dev = torch.device("cuda", int(device) if not isinstance(device, torch.device) else device.index)
    out = torch.empty((int(n), 3, 4), dtype=torch.float64, device=dev)
    m = (ctypes.c_double * 3)(*(float(x) for x in masses))
    lib = _lib.load()
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = lib.ctpwa_phase_space(float(M), m, int(n), int(seed) & (2**64 - 1), out.data_ptr(), ctypes.c_void_p(stream))
    if rc != 0:
        raise RuntimeError(_lib.error(None))
    return out


def write_dat(path, p4):
    """Reference .dat layout: one 'E px py pz' line per particle."""
    flat = np.ascontiguousarray(p4, dtype=np.float64).reshape(-1, 4)
    np.savetxt(path, flat, fmt="%.17g")


def write_npy(path, p4):
    np.save(path, np.ascontiguousarray(p4, dtype=np.float64))


def accept_reject(p4, intensity, seed, safety=1.2, n_max=None):
    """Keep events with probability intensity / (safety * max(intensity))."""
    rng = np.random.default_rng(seed)
    I = np.asarray(intensity, dtype=np.float64)
    imax = safety * float(np.max(I))
    keep = rng.uniform(0.0, imax, I.size) < I
    sel = p4[keep]
    if n_max is not None:
        sel = sel[:n_max]
    return sel
