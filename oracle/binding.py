"""ctypes binding of the CPU oracle (oracle/liboracle.so) and of the
reference-math shim (oracle/_ref/libref_math.so).

Test infrastructure: used by tests/, by the smoke check and by the CPU
baseline leg of bench.py, never by the product path."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libref_math.so")
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)

_orc = None


def oracle_lib():
    global _orc
    if _orc is None:
        lib = ctypes.CDLL(ORACLE_SO)
        lib.orc_open.restype = ctypes.c_void_p
        lib.orc_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        lib.orc_open_shard.restype = ctypes.c_void_p
        lib.orc_open_shard.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        lib.orc_shard_sums.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_int]
        lib.orc_finalize_sums.argtypes = [ctypes.c_void_p, _D, _D, _D, _D]
        lib.orc_close.argtypes = [ctypes.c_void_p]
        lib.orc_sizes.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]
        lib.orc_theta_init.argtypes = [ctypes.c_void_p, _D]
        lib.orc_group_nsl.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.orc_slamp.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D]
        lib.orc_columns.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D]
        lib.orc_nll_grad.argtypes = [ctypes.c_void_p, _D, _D, _D, _D, ctypes.c_int]
        lib.orc_pwa_amp.argtypes = [_D, ctypes.c_int, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D]
        lib.orc_clebsch.restype = ctypes.c_double
        lib.orc_clebsch.argtypes = [ctypes.c_int] * 6
        lib.orc_small_d.restype = ctypes.c_double
        lib.orc_small_d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        lib.orc_ylm.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, _D]
        lib.orc_custom_eval.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _D, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, _D, ctypes.c_char_p, ctypes.c_int]
        lib.orc_model_eval.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, _D,
                                       _I, _D, ctypes.c_int, _D, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double, _D]
        lib.orc_intensity.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D]
        lib.orc_take.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_long), ctypes.c_long]
        lib.orc_error.restype = ctypes.c_char_p
        lib.orc_error.argtypes = [ctypes.c_void_p]
        _orc = lib
    return _orc


def ref_lib():
    if not os.path.exists(REF_SO):
        return None
    lib = ctypes.CDLL(REF_SO)
    V = ctypes.c_void_p
    lib.ref_pwa_amp.argtypes = [_D, ctypes.c_int, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D]
    lib.ref_clebsch.restype = ctypes.c_double
    lib.ref_clebsch.argtypes = [ctypes.c_int] * 6
    lib.ref_model_build.restype = V
    lib.ref_model_build.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_int, _D, _I, _D, ctypes.c_int]
    lib.ref_custom_build.restype = V
    lib.ref_custom_build.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    lib.ref_aux_eval.argtypes = [V, _D, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_double, _D, _D]
    lib.ref_aux_free.argtypes = [V]
    return lib


def ptr(a):
    return a.ctypes.data_as(_D)


class Oracle:
    """FP64 CPU oracle of one config (test infrastructure)."""

    def __init__(self, config_path, shard=None):
        self.lib = oracle_lib()
        err = ctypes.create_string_buffer(1024)
        rank, world = (0, 1) if shard is None else shard
        self.h = self.lib.orc_open_shard(str(config_path).encode(), int(rank), int(world), err, 1024)
        if not self.h:
            raise RuntimeError("oracle: " + err.value.decode())
        sz = (ctypes.c_long * 8)()
        self.lib.orc_sizes(self.h, sz)
        self.nA, self.nT, self.nV, self.npol, self.nG = sz[0], sz[1], sz[2], sz[3], sz[4]
        self.nev = (sz[5], sz[6], sz[7])

    def close(self):
        if self.h:
            self.lib.orc_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _params(self, params):
        """The parameter array as the C side reads it: 2 nV + nT doubles
        (a shorter array would be read past its end)."""
        p = np.ascontiguousarray(params, dtype=np.float64)
        if p.ndim != 1 or p.size != 2 * self.nV + self.nT:
            raise ValueError(f"params: expected {2 * self.nV + self.nT} values, got shape {p.shape}")
        return p

    def nll_grad(self, params, nthreads=0):
        p = self._params(params)
        g = np.zeros_like(p)
        v = ctypes.c_double()
        parts = np.zeros(6)
        rc = self.lib.orc_nll_grad(self.h, ptr(p), ctypes.byref(v), ptr(g), ptr(parts), nthreads)
        if rc != 0:
            raise RuntimeError(self.lib.orc_error(self.h).decode())
        return v.value, g, parts

    def shard_sums(self, params, nthreads=0):
        """Per-sample sums of this oracle's events (layout of the engine's shard sums)."""
        p = self._params(params)
        out = np.zeros(3 * (2 + 2 * self.nA + self.nT) + 4)
        if self.lib.orc_shard_sums(self.h, ptr(p), ptr(out), nthreads) != 0:
            raise RuntimeError(self.lib.orc_error(self.h).decode())
        return out

    def finalize_sums(self, params, sums):
        """(nll, grad) from summed shard sums."""
        p = self._params(params)
        s = np.ascontiguousarray(sums, dtype=np.float64)
        g = np.zeros_like(p)
        v = ctypes.c_double()
        if self.lib.orc_finalize_sums(self.h, ptr(p), ptr(s), ctypes.byref(v), ptr(g)) != 0:
            raise RuntimeError(self.lib.orc_error(self.h).decode())
        return v.value, g

    def theta_init(self):
        """[3, nT]: initial value, lower and upper bound of every free resonance parameter."""
        out = np.zeros((3, self.nT))
        self.lib.orc_theta_init(self.h, ptr(out))
        return out

    def columns(self, kind, theta):
        t = np.ascontiguousarray(theta, dtype=np.float64)
        if t.ndim != 1 or t.size != self.nT:
            raise ValueError(f"theta: expected {self.nT} values, got shape {t.shape}")
        out = np.zeros((self.nev[kind], self.npol, self.nA), dtype=np.complex128)
        self.lib.orc_columns(self.h, kind, ptr(t), out.ctypes.data_as(_D))
        return out

    def take(self, kind, idx):
        """Replace sample `kind` by its events idx (repeats allowed), keeping
        their computed angular tensors."""
        ix = np.ascontiguousarray(idx, dtype=np.int64)
        if self.lib.orc_take(self.h, int(kind), ix.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), ix.size) != 0:
            raise RuntimeError(self.lib.orc_error(self.h).decode())
        nev = list(self.nev)
        nev[kind] = int(ix.size)
        self.nev = tuple(nev)

    def intensity(self, kind, params):
        p = self._params(params)
        out = np.zeros(self.nev[kind])
        self.lib.orc_intensity(self.h, kind, ptr(p), ptr(out))
        return out

    # ---- second derivatives (checkers for the device Hessian) ----
    # Richardson-extrapolated central differences of the oracle's exact
    # (dual-number) gradient and of its per-sample sums: D(h) = (f(x+h) -
    # f(x-h)) / 2h, R = (4 D(h/2) - D(h)) / 3. Steps are rel * max(|p_i|, 1e-2):
    # with rel = 1e-5 a mass step stays ~1e-3 of a resonance width, and two
    # step sizes agree to ~2e-10 of the largest Hessian entry (K+K-pi0).

    @staticmethod
    def _richardson(f, x, u, eps):
        def d(h):
            return (f(x + h * u) - f(x - h * u)) / (2 * h)

        return (4 * d(eps / 2) - d(eps)) / 3

    @staticmethod
    def _step(p, u, rel):
        m = np.abs(u) > 0
        return rel * float(np.min(np.maximum(np.abs(p[m]), 1e-2) / np.abs(u[m])))

    def hessian_fd(self, params, rel=1e-5):
        """[nP, nP] Hessian of the oracle NLL (symmetrised)."""
        p = self._params(params)
        n = p.size
        H = np.zeros((n, n))
        for i in range(n):
            u = np.zeros(n)
            u[i] = 1.0
            H[i] = self._richardson(lambda q: self.nll_grad(q)[1], p, u, self._step(p, u, rel))
        return 0.5 * (H + H.T)

    def hvp_sums_fd(self, params, dirs, rel=1e-5):
        """[ndir, 3 nacc] directional derivatives of shard_sums' per-sample sums."""
        p = self._params(params)
        nacc = 2 + 2 * self.nA + self.nT
        out = []
        for u in np.atleast_2d(dirs):
            out.append(self._richardson(lambda q: self.shard_sums(q)[:3 * nacc], p, u, self._step(p, u, rel)))
        return np.array(out)

    def finalize_hvp_fd(self, params, dirs, sums, tsums, rel=1e-5):
        """[ndir, nP] rows H u from value sums and tangent sums: the directional
        derivative of finalize_sums along (u, tangent sums)."""
        p = self._params(params)
        s = np.ascontiguousarray(sums, dtype=np.float64)
        nacc = 2 + 2 * self.nA + self.nT
        dirs = np.atleast_2d(dirs)
        tsums = np.asarray(tsums, dtype=np.float64).reshape(len(dirs), 3 * nacc)
        out = []
        for u, t in zip(dirs, tsums):
            x = np.concatenate([p, s])
            w = np.concatenate([u, t, np.zeros(s.size - 3 * nacc)])

            def f(y):
                return self.finalize_sums(y[:p.size], y[p.size:])[1]

            out.append(self._richardson(f, x, w, self._step(p, u, rel)))
        return np.array(out)
