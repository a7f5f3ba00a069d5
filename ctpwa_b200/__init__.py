"""ctpwa_b200 — B200-native event-parallel likelihood engine for partial-wave analysis.

Drop-in for the reference module ``ctpwa`` (pybind11 class ``analysis``,
src/main.cu:91-131)::

    import ctpwa_b200 as ctpwa
    ana = ctpwa.analysis("config.yml")
    p = torch.tensor(..., dtype=torch.float64, device="cuda")  # [2*nV + nT]
    p.requires_grad_(True)
    nll = ana.getNLL(p)            # 0-d float64 CUDA tensor, differentiable
    g, = torch.autograd.grad(nll, p)
    H = ana.getHessian(p)          # [(2nV+nT), (2nV+nT)] float64 CUDA

Parameter layout, names and defaults follow the reference
(``getNVector``, ``getNFreeTheta``, ``getParamNames``, ``getFreeResParams``).
Everything runs through the C ABI of ``libctpwa_b200.so`` (include/ctpwa_b200.h);
there is no CPU path.
"""
from __future__ import annotations

import ctypes
import json
import warnings

import torch

from . import _lib

__all__ = ["analysis", "DecayInfo", "EvalBatch", "describe", "precompile", "spd_inverse", "version"]

_PRECISIONS = {"fp64": 0, "double": 0, "plain": 0, "mixed": 1, "fp32": 1, "float": 1}


def version() -> str:
    return _lib.load().ctpwa_version().decode()


def precompile(config_file: str) -> float:
    """Compile the fused kernel of a config's model into the kernel cache (no GPU needed)."""
    lib = _lib.load()
    sec = ctypes.c_double(0.0)
    err = ctypes.create_string_buffer(4096)
    rc = lib.ctpwa_precompile(str(config_file).encode(), ctypes.byref(sec), err, 4096)
    if rc != 0:
        raise RuntimeError(err.value.decode("utf-8", "replace"))
    return sec.value


def spd_inverse(a: torch.Tensor) -> torch.Tensor:
    """Inverse of a symmetric positive definite float64 CUDA matrix, computed
    on its device in FP64 (C ABI ctpwa_spd_inverse). Raises RuntimeError when
    the matrix is not positive definite."""
    if a.dim() != 2 or a.shape[0] != a.shape[1] or a.dtype != torch.float64 or not a.is_cuda:
        raise RuntimeError("spd_inverse expects a square float64 CUDA matrix")
    a = a.contiguous()
    out = torch.empty_like(a)
    info = torch.zeros(1, dtype=torch.int32, device=a.device)
    stream = torch.cuda.current_stream(a.device).cuda_stream
    lib = _lib.load()
    if lib.ctpwa_spd_inverse(a.data_ptr(), a.shape[0], out.data_ptr(), info.data_ptr(), ctypes.c_void_p(stream)) != 0:
        raise RuntimeError(_lib.error(None))
    k = int(info.item())
    if k:
        raise RuntimeError(f"matrix is not positive definite (pivot {k})")
    return out


class EvalBatch:
    """Several analyses of one model evaluated in one launch (C ABI
    ctpwa_batch_*): ``nll_grad`` for device parameters of several jobs at
    once, and ``analysis.fit(..., batch=b)`` for fits on several threads whose
    evaluations are gathered into shared launches (serving)."""

    def __init__(self, device: int = 0):
        self._lib = _lib.load()
        self._b = self._lib.ctpwa_batch_create(int(device))
        if not self._b:
            raise RuntimeError(_lib.error(None))
        self.device = int(device)

    def close(self):
        if getattr(self, "_b", None):
            self._lib.ctpwa_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        self.close()

    def nll_grad(self, analyses, params, precision="fp64"):
        """[(nll, grad)] of each analysis at its float64 CUDA parameters, one launch per stage for all."""
        n = len(analyses)
        ps = [a._check_params(p) for a, p in zip(analyses, params)]
        nll = [torch.empty((), dtype=torch.float64, device=p.device) for p in ps]
        grad = [torch.empty_like(p) for p in ps]
        VP = ctypes.c_void_p * n
        hs = VP(*[a._h for a in analyses])
        dp, dn, dg = VP(*[p.data_ptr() for p in ps]), VP(*[x.data_ptr() for x in nll]), VP(*[x.data_ptr() for x in grad])
        stream = torch.cuda.current_stream(ps[0].device).cuda_stream if n else 0
        prec = analysis._parse_precision(precision)
        if self._lib.ctpwa_nll_grad_multi(self._b, hs, n, dp, dn, dg, prec, ctypes.c_void_p(stream)) != 0:
            raise RuntimeError(_lib.error(None))
        return list(zip(nll, grad))

    def stats(self):
        """(rounds, requests) of the gathered host evaluations so far."""
        r, q = ctypes.c_longlong(0), ctypes.c_longlong(0)
        self._lib.ctpwa_batch_stats(self._b, ctypes.byref(r), ctypes.byref(q))
        return r.value, q.value


def describe(config_file: str) -> dict:
    """Lowered model of a config (no GPU needed): amplitude columns, groups,
    resonance blocks, theta slots, coupling map and parameter names."""
    lib = _lib.load()
    err = ctypes.create_string_buffer(4096)
    n = lib.ctpwa_describe(str(config_file).encode(), None, 0, err, 4096)
    if n < 0:
        raise RuntimeError(err.value.decode("utf-8", "replace"))
    buf = ctypes.create_string_buffer(n)
    lib.ctpwa_describe(str(config_file).encode(), buf, n, err, 4096)
    return json.loads(buf.value.decode("utf-8"))


class DecayInfo:
    """Host-side model information of a config (reference ``ctpwa.DecayInfo``)."""

    def __init__(self, config_file: str = "config.yml"):
        try:
            self._m = describe(config_file)
        except RuntimeError as e:
            if "analysis not initialized" not in str(e):
                raise
            self._m = None

    def isValid(self) -> bool:
        return self._m is not None

    def nAmplitudes(self) -> int:
        return len(self._m["amplitude_names"])

    def amplitudeNames(self):
        return list(self._m["amplitude_names"])

    def resonanceParamNames(self):
        return [s["name"] for s in self._m["slots"]]

    def resonanceNames(self):
        names = []
        for b in self._m["blocks"]:
            g = self._m["groups"][b["group"]]
            rep = {r["tag"]: r["name"] for r in b["res"]}
            names.append("_".join(
                f"{rep.get(g['particles'][n['mother']], g['particles'][n['mother']])}\u2192"
                f"{rep.get(g['particles'][n['d1']], g['particles'][n['d1']])}+"
                f"{rep.get(g['particles'][n['d2']], g['particles'][n['d2']])}" for n in g["nodes"]))
        return names

    def hasCouplingMatrix(self) -> bool:
        return True

    def print(self):
        print("=== DecayInfo ===")
        print(f"Amplitudes: {self.nAmplitudes()}")
        for i, n in enumerate(self.amplitudeNames()):
            print(f"  [{i}] {n}")
        print(f"Resonance theta params ({len(self._m['slots'])}):")
        for i, n in enumerate(self.resonanceParamNames()):
            print(f"  [{i}] {n}")


class _NLLFunction(torch.autograd.Function):
    """Forward evaluates the NLL and its gradient in one device pass; backward
    returns the stored gradient times the incoming grad (reference
    NLLFunction, src/Analysis.cu:625-1261)."""

    @staticmethod
    def forward(ctx, params, ana):
        nll, grad = ana._eval(params)
        ctx.save_for_backward(grad)
        return nll

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return grad * grad_out, None


class analysis:
    """Likelihood of one config.yml model over its phase-space, data and
    background samples (reference ``ctpwa.analysis``)."""

    def __init__(self, config_file: str = "config.yml", device=None, precision: str = "fp64", shard=None):
        """shard=(rank, world) keeps event block `rank` of `world` of every
        sample (multi-GPU event sharding; see getShardSums)."""
        self._h = None
        self._lib = _lib.load()
        if device is None:
            device = torch.cuda.current_device() if torch.cuda.is_available() else 0
        self._device = int(device)
        self._precision = self._parse_precision(precision)
        self._fit_mode = 1
        status = ctypes.c_int(0)
        err = ctypes.create_string_buffer(4096)
        rank, world = (0, 1) if shard is None else (int(shard[0]), int(shard[1]))
        self._shard = (rank, world)
        h = self._lib.ctpwa_create_shard(str(config_file).encode(), self._device, rank, world, ctypes.byref(status),
                                         err, 4096)
        if not h:
            msg = err.value.decode("utf-8", "replace")
            if status.value == -1 and msg.startswith("analysis not initialized"):
                # reference: warning + isValid() == False, later calls raise
                warnings.warn(f'Config file "{config_file}" is empty or not found. Analysis not initialized. ({msg})')
                return
            raise RuntimeError(msg)
        self._h = ctypes.c_void_p(h)
        self._np = self._lib.ctpwa_n_params(self._h)

    @classmethod
    def from_device(cls, config_file: str, phsp, data, bkg=None, weights=None, device=None,
                    precision: str = "fp64", fp64_only: bool = False) -> "analysis":
        """Analysis over in-memory samples: the model from config_file, the
        events from float64 CUDA tensors [n, n_final, 4] (E, px, py, pz in the
        config's Data.order) instead of the config's Data files. weights: None
        or three per-event float64 CUDA tensors / None (phase space, data,
        background). The tensors are copied; pending work on the current
        stream is waited for first. fp64_only: build neither the mixed-form
        tables nor the polarisation pairing (FP64 evaluations and intensities
        only; cheaper to build)."""
        self = cls.__new__(cls)
        self._h = None
        self._lib = _lib.load()
        if device is None:
            device = phsp.device.index if phsp.is_cuda else torch.cuda.current_device()
        self._device = int(device)
        self._precision = self._parse_precision(precision)
        self._fit_mode = 1
        self._shard = (0, 1)
        samples = [phsp, data, bkg]
        ws = list(weights) if weights is not None else [None, None, None]
        keep = []
        p4 = (ctypes.c_void_p * 3)()
        n = (ctypes.c_longlong * 3)()
        w = (ctypes.c_void_p * 3)()
        for k, t in enumerate(samples):
            if t is None:
                continue
            if t.dtype != torch.float64 or not t.is_cuda or t.dim() != 3 or t.shape[2] != 4:
                raise RuntimeError("in-memory samples must be float64 CUDA tensors [n, n_final, 4]")
            if t.device.index != self._device:
                raise RuntimeError(f"in-memory samples must be on cuda:{self._device}")
            t = t.contiguous()
            keep.append(t)
            p4[k] = t.data_ptr()
            n[k] = t.shape[0]
            if ws[k] is not None:
                wt = ws[k].to(device=t.device, dtype=torch.float64).contiguous()
                if wt.numel() != t.shape[0]:
                    raise RuntimeError("one weight per event")
                keep.append(wt)
                w[k] = wt.data_ptr()
        torch.cuda.current_stream(self._device).synchronize()
        status = ctypes.c_int(0)
        err = ctypes.create_string_buffer(4096)
        h = self._lib.ctpwa_create_from_device_flags(str(config_file).encode(), self._device, p4, n, w,
                                                     1 if fp64_only else 0, ctypes.byref(status), err, 4096)
        if not h:
            raise RuntimeError(err.value.decode("utf-8", "replace"))
        self._h = ctypes.c_void_p(h)
        self._np = self._lib.ctpwa_n_params(self._h)
        return self

    # ------------------------------------------------------------ lifecycle
    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h is not None:
            try:
                # the handle's memory goes back to the pool without waiting
                # for other streams: let work queued on the current one finish
                torch.cuda.current_stream(self._device).synchronize()
                self._lib.ctpwa_destroy(h)
            except Exception:
                pass

    def isValid(self) -> bool:
        return self._h is not None

    def _check(self):
        if self._h is None:
            raise RuntimeError("analysis not initialized: invalid or missing config file")

    @staticmethod
    def _parse_precision(p):
        if isinstance(p, int):
            if p not in (0, 1):
                raise ValueError("precision must be 'fp64' or 'mixed'")
            return p
        try:
            return _PRECISIONS[str(p).lower()]
        except KeyError:
            raise ValueError("precision must be 'fp64' or 'mixed'") from None

    def setPrecision(self, precision):
        """'fp64' (plain FP64, the drop-in default) or 'mixed' (FP32 amplitudes, FP64 reductions)."""
        self._precision = self._parse_precision(precision)

    def getPrecision(self) -> str:
        return "mixed" if self._precision == 1 else "fp64"

    # ------------------------------------------------------------ counts/names
    def setFitMode(self, mode: int):
        if int(mode) != 1:
            raise RuntimeError("only fit mode 1 (vspace couplings, the reference default) is supported")
        self._fit_mode = 1

    def getFitMode(self) -> int:
        return self._fit_mode

    def getNVector(self) -> int:
        self._check()
        return self._lib.ctpwa_n_vector(self._h)

    def getNFreeTheta(self) -> int:
        self._check()
        return self._lib.ctpwa_n_free_theta(self._h)

    def getNParams(self) -> int:
        self._check()
        return self._np

    def getParamNames(self):
        self._check()
        s = _lib.read_string(self._lib.ctpwa_param_names, self._h)
        return s.split("\n") if s else []

    def getFreeResParams(self) -> torch.Tensor:
        """CPU float64 tensor [3, nT]: initial values, lower and upper bounds."""
        self._check()
        nt = self.getNFreeTheta()
        out = torch.empty((3, nt), dtype=torch.float64)
        if nt:
            rc = self._lib.ctpwa_free_res_params(self._h, ctypes.cast(out.data_ptr(), ctypes.POINTER(ctypes.c_double)))
            if rc != 0:
                raise RuntimeError(_lib.error(self._h))
        return out

    def getModel(self) -> dict:
        """Lowered model (amplitude columns, groups, theta slots, coupling map)."""
        self._check()
        return json.loads(_lib.read_string(self._lib.ctpwa_model_json, self._h))

    def getNEvents(self):
        self._check()
        return tuple(int(self._lib.ctpwa_n_events(self._h, k)) for k in range(3))

    def getAmplitudeNames(self):
        self._check()
        return list(self.getModel()["amplitude_names"])

    def getNPolarizations(self) -> int:
        self._check()
        return int(self.getModel()["npol"])

    def getSLVectors(self) -> torch.Tensor:
        """Number of SL combinations per resonance block (int32, CUDA)."""
        m = self.getModel()
        nsl = [len(m["groups"][b["group"]]["sl_combs"]) for b in m["blocks"]]
        return torch.tensor(nsl, dtype=torch.int32, device=f"cuda:{self._device}")

    def deviceBytes(self) -> int:
        self._check()
        return int(self._lib.ctpwa_device_bytes(self._h))

    # ------------------------------------------------------------ evaluation
    def _check_params(self, params: torch.Tensor) -> torch.Tensor:
        self._check()
        if not isinstance(params, torch.Tensor) or params.dtype != torch.float64:
            raise RuntimeError("params must be float64")
        if not params.is_cuda or params.device.index != self._device:
            raise RuntimeError(f"params must be on the primary GPU (cuda:{self._device}), got {params.device}")
        if params.dim() != 1:
            raise RuntimeError("params must be 1-dimensional")
        if params.numel() != self._np:
            raise RuntimeError(f"params size mismatch: got {params.numel()}, expected {self._np}")
        return params.detach().contiguous()

    def _eval(self, params: torch.Tensor, precision=None, cached=False):
        p = self._check_params(params)
        nll = torch.empty((), dtype=torch.float64, device=p.device)
        grad = torch.empty_like(p)
        stream = torch.cuda.current_stream(p.device).cuda_stream
        prec = self._precision if precision is None else self._parse_precision(precision)
        fn = self._lib.ctpwa_nll_grad_cached if cached else self._lib.ctpwa_nll_grad
        rc = fn(self._h, p.data_ptr(), nll.data_ptr(), grad.data_ptr(), prec, ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError(_lib.error(self._h))
        return nll, grad

    def getNLL(self, params: torch.Tensor) -> torch.Tensor:
        """Negative log-likelihood (0-d float64 CUDA tensor); differentiable."""
        self._check_params(params)
        return _NLLFunction.apply(params, self)

    def getNLLAndGrad(self, params: torch.Tensor, precision=None, cached=False):
        """(nll, grad) without autograd bookkeeping. cached=True: from the
        normalisation cache (cacheNormalisation), which must have been built
        at the same resonance parameters; the phase-space sample is not read."""
        return self._eval(params, precision, cached)

    def cacheNormalisation(self, params: torch.Tensor) -> float:
        """Build the normalisation cache at the resonance parameters of
        `params`: the phase-space sums as FP64 quadratic forms in the
        couplings, with the lineshape derivatives (the reference keeps its
        phase-space matrix between evaluations when no resonance parameter is
        free, src/Analysis.cu:748-829). Afterwards host-buffer evaluations
        (getNLLHost, fit, fitNewton) at these resonance parameters, and
        getNLLAndGrad(cached=True), read only the data and background samples.
        The fits build the cache themselves when no resonance parameter is
        free. Returns the device time of the phase-space pass in ms."""
        p = self._check_params(params)
        ms = ctypes.c_double()
        stream = torch.cuda.current_stream(p.device).cuda_stream
        if self._lib.ctpwa_norm_cache_build(self._h, p.data_ptr(), ctypes.byref(ms), ctypes.c_void_p(stream)) != 0:
            raise RuntimeError(_lib.error(self._h))
        return ms.value

    def clearNormalisationCache(self):
        """Drop the normalisation cache (every evaluation takes the full pass again)."""
        self._check()
        self._lib.ctpwa_norm_cache_clear(self._h)

    def hasNormalisationCache(self) -> bool:
        self._check()
        return bool(self._lib.ctpwa_norm_cache_valid(self._h))

    def getNLLHost(self, params, precision=None):
        """Evaluate from host memory through the C ABI's host-buffer entry point."""
        self._check()
        import numpy as np

        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64))
        if p.size != self._np:
            raise RuntimeError(f"params size mismatch: got {p.size}, expected {self._np}")
        g = np.empty_like(p)
        v = ctypes.c_double()
        dp = ctypes.POINTER(ctypes.c_double)
        prec = self._precision if precision is None else self._parse_precision(precision)
        rc = self._lib.ctpwa_nll_grad_host(self._h, p.ctypes.data_as(dp), ctypes.byref(v), g.ctypes.data_as(dp),
                                           prec, None)
        if rc != 0:
            raise RuntimeError(_lib.error(self._h))
        return v.value, g

    def fit(self, start, lower=None, upper=None, free=None, max_evals=100, history=20, ftol=1e-13, gtol=1e-9,
            precision=None, stream=None, batch=None):
        """Minimise the NLL from `start` (host array of all parameters) by the
        library's projected limited-memory BFGS (``ctpwa_fit``), one
        host-buffer evaluation per function call, the whole loop in native
        code on this thread (the GIL is released meanwhile).

        Defaults follow the reference's fit (example/fit.py:113-160): the
        first coupling (real and imaginary part) stays fixed, the couplings are
        unbounded and the free resonance parameters stay within their bounds
        (getFreeResParams). `lower` / `upper` / `free` (length n_params)
        replace those defaults. Returns (params, nll, evaluations, iterations,
        status, eval_ms); status 0: projected gradient <= gtol, 1: relative
        decrease <= ftol, 2: max_evals spent, 3: no decrease found. With
        `batch` (an EvalBatch), every evaluation is gathered with those of the
        other fits running in the batch (one launch for all of them). Without
        `batch`, when no resonance parameter can move (free 0 or lower ==
        upper for all of them), the fit builds the normalisation cache
        (cacheNormalisation) and its evaluations read only the data and
        background samples."""
        self._check()
        import numpy as np

        x, lo, hi, fr = self._fit_box(start, lower, upper, free)
        out = np.zeros(4)
        lat = np.zeros(max(1, int(max_evals)), dtype=np.float32)
        dp = ctypes.POINTER(ctypes.c_double)
        prec = self._precision if precision is None else self._parse_precision(precision)
        sp = None if stream is None else ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else stream)
        if batch is not None:
            rc = self._lib.ctpwa_fit_batched(batch._b, self._h, x.ctypes.data_as(dp),
                                             fr.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), lo.ctypes.data_as(dp),
                                             hi.ctypes.data_as(dp), prec, int(max_evals), int(history), float(ftol),
                                             float(gtol), out.ctypes.data_as(dp),
                                             lat.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        else:
            rc = self._lib.ctpwa_fit(self._h, x.ctypes.data_as(dp), fr.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                                     lo.ctypes.data_as(dp), hi.ctypes.data_as(dp), prec, int(max_evals), int(history),
                                     float(ftol), float(gtol), out.ctypes.data_as(dp),
                                     lat.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), sp)
        if rc != 0:
            raise RuntimeError(_lib.error(self._h))
        ne = int(out[1])
        return x, float(out[0]), ne, int(out[2]), int(out[3]), lat[:min(ne, lat.size)].astype(np.float64).tolist()

    def _fit_box(self, start, lower, upper, free):
        """Start (copied), bounds and free mask of a fit, with the reference's
        defaults (example/fit.py:113-160): the first coupling fixed, the
        couplings unbounded, the free resonance parameters within their
        bounds."""
        import numpy as np

        n = self._np
        x = np.ascontiguousarray(np.asarray(start, dtype=np.float64)).copy()
        if x.size != n:
            raise RuntimeError(f"params size mismatch: got {x.size}, expected {n}")
        nV = self.getNVector()
        if lower is None or upper is None:
            res = self.getFreeResParams().numpy()
            lo = np.concatenate([np.full(2 * nV, -np.inf), res[1]])
            hi = np.concatenate([np.full(2 * nV, np.inf), res[2]])
            lower = lo if lower is None else lower
            upper = hi if upper is None else upper
        lo = np.ascontiguousarray(lower, dtype=np.float64)
        hi = np.ascontiguousarray(upper, dtype=np.float64)
        if free is None:
            free = np.ones(n, dtype=np.uint8)
            free[0] = free[nV] = 0
        fr = np.ascontiguousarray(free, dtype=np.uint8)
        if lo.size != n or hi.size != n or fr.size != n:
            raise RuntimeError("fit: lower, upper and free need n_params entries")
        return x, lo, hi, fr

    def fitNewton(self, start, lower=None, upper=None, free=None, max_iter=50, xtol=1e-4, gtol=1e-9, fnoise=None,
                  precision=None, stream=None):
        """Newton fit with the exact FP64 Hessian (``ctpwa_fit_newton``):
        Levenberg-Marquardt steps over the same box and free parameters as
        `fit`, converging to the stationary point of the start's basin (the
        reference keeps a fit result only where its Hessian is positive
        definite, example/fit.py:202-230). The NLL and gradient are taken in
        `precision`; the Hessian is FP64 in both forms. Stops after a step of
        at most `xtol` in units of 1/sqrt(H_ii) per parameter, or one whose
        predicted decrease is below 1e-2 `fnoise`. `fnoise` is the NLL's
        rounding level (default 1e-3 for the mixed form, 1e-6 for FP64):
        steps predicted to gain less are accepted unless the NLL rises by more.
        Returns (params, nll, evaluations, hessians, status); status 0:
        projected gradient <= gtol, 1: step <= xtol, 2: max_iter Hessians
        spent, 3: no acceptable step."""
        self._check()
        import numpy as np

        x, lo, hi, fr = self._fit_box(start, lower, upper, free)
        prec = self._precision if precision is None else self._parse_precision(precision)
        if fnoise is None:
            fnoise = 1e-3 if prec == 1 else 1e-6
        out = np.zeros(4)
        dp = ctypes.POINTER(ctypes.c_double)
        sp = None if stream is None else ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else stream)
        rc = self._lib.ctpwa_fit_newton(self._h, x.ctypes.data_as(dp), fr.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                                        lo.ctypes.data_as(dp), hi.ctypes.data_as(dp), prec, int(max_iter), float(xtol),
                                        float(gtol), float(fnoise), out.ctypes.data_as(dp), sp)
        if rc != 0:
            raise RuntimeError(_lib.error(self._h))
        return x, float(out[0]), int(out[1]), int(out[2]), int(out[3])

    def getShardSums(self, params: torch.Tensor, precision=None) -> torch.Tensor:
        """This shard's per-sample sums (float64 CUDA, to be summed over shards
        with one all-reduce and passed to finalizeShardSums)."""
        p = self._check_params(params)
        out = torch.empty(self._lib.ctpwa_sums_size(self._h), dtype=torch.float64, device=p.device)
        stream = torch.cuda.current_stream(p.device).cuda_stream
        prec = self._precision if precision is None else self._parse_precision(precision)
        if self._lib.ctpwa_shard_sums(self._h, p.data_ptr(), prec, out.data_ptr(), ctypes.c_void_p(stream)) != 0:
            raise RuntimeError(_lib.error(self._h))
        return out

    def finalizeShardSums(self, params: torch.Tensor, sums: torch.Tensor):
        """(nll, grad) of the union of the shards from the summed shard sums."""
        p = self._check_params(params)
        if sums.dtype != torch.float64 or not sums.is_cuda or sums.numel() != self._lib.ctpwa_sums_size(self._h):
            raise RuntimeError("sums must be the float64 CUDA buffer of getShardSums")
        sums = sums.contiguous()
        nll = torch.empty((), dtype=torch.float64, device=p.device)
        grad = torch.empty_like(p)
        stream = torch.cuda.current_stream(p.device).cuda_stream
        if self._lib.ctpwa_finalize_sums(self._h, p.data_ptr(), sums.data_ptr(), nll.data_ptr(), grad.data_ptr(),
                                         ctypes.c_void_p(stream)) != 0:
            raise RuntimeError(_lib.error(self._h))
        return nll, grad

    def getNBlocks(self) -> int:
        """Number of resonance blocks (partial waves of the fit fractions)."""
        self._check()
        return int(self._lib.ctpwa_n_blocks(self._h))

    def getPartialIntegrals(self, params: torch.Tensor, kind: int = 0) -> torch.Tensor:
        """Per resonance block i: sum_e w_e sum_pol |sum_{a in i} v_a A_a|^2 over
        sample kind 0 (phase space), 1 (data), 2 (background) or 3
        (Data.phsp_truth). float64 CUDA [nBlocks]."""
        p = self._check_params(params)
        out = torch.empty(self.getNBlocks(), dtype=torch.float64, device=p.device)
        stream = torch.cuda.current_stream(p.device).cuda_stream
        rc = self._lib.ctpwa_partial_integrals(self._h, p.data_ptr(), int(kind), out.data_ptr(), ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError(_lib.error(self._h))
        return out

    def getFitFractions(self, params: torch.Tensor, hessian: torch.Tensor = None) -> torch.Tensor:
        """Fit fractions FF_i = I_i / sum_j I_j of the resonance blocks (reference
        analysis::getFitFractions, src/Analysis.cu:3527-3630), integrated over
        Data.phsp_truth (or over the phase-space sample when the config has no
        phsp_truth). Errors: J_FF H^-1 J_FF^T with the coupling block of the
        Hessian (`hessian` if given, else getHessian(params)) over the free
        couplings (the first coupling is the fixed reference), J_FF by central
        differences (step 5e-6 max(|p_j|, 1)). Returns CPU float64 [nBlocks, 2] =
        [center, error]; errors are 0 when the Hessian block is not positive
        definite."""
        import numpy as np

        p = self._check_params(params).clone()
        kind = 3
        try:
            self.getPartialIntegrals(p, 3)
        except RuntimeError as e:
            if "phsp_truth" not in str(e):
                raise
            kind = 0

        def ff(q):
            I = self.getPartialIntegrals(q, kind)
            tot = float(I.sum())
            return (I / (tot if tot > 0 else 1e-30)).cpu().numpy()

        center = ff(p)
        n = self.getNVector()
        free = [j for j in range(2 * n) if j not in (0, n)]
        errors = np.zeros_like(center)
        if free:
            H = hessian if hessian is not None else self.getHessian(p)
            mask = torch.zeros(self.getNParams(), dtype=torch.bool)
            mask[free] = True
            try:
                covd = self.getCovariance(p, free=mask, hessian=H)
            except RuntimeError:
                covd = None
            if covd is not None:
                cov = covd.cpu().numpy()[np.ix_(free, free)]
                J = np.zeros((center.size, len(free)))
                for c, j in enumerate(free):
                    eps = 5e-6 * max(abs(float(p[j])), 1.0)
                    qp = p.clone()
                    qp[j] += eps
                    qm = p.clone()
                    qm[j] -= eps
                    J[:, c] = (ff(qp) - ff(qm)) / (2 * eps)
                errors = np.sqrt(np.maximum(np.einsum("ij,jk,ik->i", J, cov, J), 0.0))
        return torch.tensor(np.stack([center, errors], axis=1), dtype=torch.float64)

    def writeResult(self, params: torch.Tensor, filename: str, is_saved_weight: int = 0, waves=()):
        """Fit-result export (reference analysis::writeResult, src/Analysis.cu:1355-1700)
        as a NumPy .npz file (ROOT is not available): `legends` (block names),
        `interference` (summed 2 Re(P_i conj P_j) over phase space, diagonal
        2|P_i|^2), `data_integral` (W_data - W_bkg), `phsp_integral` (sum of
        the per-event totals, of the blocks in `waves` when given) and
        `norm_factor`; with is_saved_weight=1 also per phase-space event
        `totalweight`, `weight_<block>` and `interf_<i>_<j>` (i < j), scaled
        to the data yield like the reference's TTree branches."""
        import numpy as np

        p = self._check_params(params)
        nb = self.getNBlocks()
        names = DecayInfo.__new__(DecayInfo)
        names._m = self.getModel()
        legends = names.resonanceNames()
        ld = int(self._lib.ctpwa_table_stride(self._h, 0))
        n = self.getNEvents()[0]
        npair = nb * (nb + 1) // 2
        dev = p.device
        total = torch.empty(ld, dtype=torch.float64, device=dev)
        partial = torch.empty(nb * ld, dtype=torch.float64, device=dev)
        interf = torch.empty(npair, dtype=torch.float64, device=dev)
        interf_ev = torch.empty(max(1, nb * (nb - 1) // 2) * ld, dtype=torch.float64, device=dev) \
            if is_saved_weight else None
        mask = None
        if waves:
            for w in waves:
                if not 0 <= int(w) < nb:
                    raise RuntimeError(f"waves index out of range: {w} (partials = {nb})")
            mask = (ctypes.c_int * nb)(*[1 if i in set(int(w) for w in waves) else 0 for i in range(nb)])
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = self._lib.ctpwa_export_weights(self._h, p.data_ptr(), mask, total.data_ptr(), partial.data_ptr(),
                                            interf_ev.data_ptr() if interf_ev is not None else None,
                                            interf.data_ptr(), ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError(_lib.error(self._h))
        # data yield: sum of data weights minus the background weight sum
        self._eval(p, 0)
        parts = self.lastParts()
        W_data, W_bkg, n_bkg = parts[3], parts[4], self.getNEvents()[2]
        data_integral = W_data - (W_bkg if W_bkg > 0 else n_bkg) if n_bkg > 0 else W_data
        tot = total[:n].cpu().numpy()
        phsp_integral = float(tot.sum())
        norm = data_integral / phsp_integral if phsp_integral != 0 else 0.0
        packed = interf.cpu().numpy()
        M = np.zeros((nb, nb))
        for i in range(nb):
            for j in range(i, nb):
                M[i, j] = M[j, i] = packed[i * nb - i * (i - 1) // 2 + (j - i)]
        out = {"legends": np.array(legends), "interference": M, "data_integral": data_integral,
               "phsp_integral": phsp_integral, "norm_factor": norm}
        if is_saved_weight:
            out["totalweight"] = tot * norm
            part = partial.view(nb, ld)[:, :n].cpu().numpy() * norm
            for i in range(nb):
                out[f"weight_{i}"] = part[i]
            ev = interf_ev.view(-1, ld)[:, :n].cpu().numpy() * norm
            k = 0
            for i in range(nb):
                for j in range(i + 1, nb):
                    out[f"interf_{i}_{j}"] = ev[k]
                    k += 1
        np.savez(filename, **out)
        return out

    def getIntensity(self, params: torch.Tensor, kind: int = 1) -> torch.Tensor:
        """Per-event intensities (float64 CUDA [n]) of sample kind 0 = phase space, 1 = data, 2 = background."""
        p = self._check_params(params)
        n = self.getNEvents()[kind]
        out = torch.empty(n, dtype=torch.float64, device=p.device)
        stream = torch.cuda.current_stream(p.device).cuda_stream
        rc = self._lib.ctpwa_intensity(self._h, p.data_ptr(), int(kind), out.data_ptr(), ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError(_lib.error(self._h))
        return out

    def getSetupTimes(self) -> dict:
        """Host milliseconds of this handle's set-up phases (model and
        generated code, CUDA context, kernel modules, sample upload, angular
        tables and kernels, the angular pass, polarisation pairing, buffers)."""
        self._check()
        buf = ctypes.create_string_buffer(1024)
        n = self._lib.ctpwa_setup_times(self._h, buf, 1024)
        if n < 0:
            raise RuntimeError(_lib.error(self._h))
        if n > 1024:
            buf = ctypes.create_string_buffer(n)
            self._lib.ctpwa_setup_times(self._h, buf, n)
        out = {}
        for item in buf.value.decode().split(";"):
            if item:
                k, v = item.split("=")
                out[k] = float(v)
        return out

    def eventLayout(self) -> dict:
        """Per-event cache layout: angular planes, polarisations, kinematic values,
        invariant masses, and the frontier values each evaluation reads (FP64
        plain path; FP32 and FP64 values of the mixed form)."""
        self._check()
        out = (ctypes.c_int * 4)()
        if self._lib.ctpwa_event_layout(self._h, out) != 0:
            raise RuntimeError(_lib.error(self._h))
        ev = (ctypes.c_int * 3)()
        if self._lib.ctpwa_event_cache_layout(self._h, ev) != 0:
            raise RuntimeError(_lib.error(self._h))
        return {"planes": out[0], "npol": out[1], "nkin": out[2], "nmass": out[3], "nev64": ev[0], "nevf": ev[1],
                "nevd": ev[2]}

    def launchShape(self) -> dict:
        """Launch shape of the fused kernels per precision: threads per CTA,
        minimum resident CTAs per SM, table staging mode, gradient sums in
        shared memory, dynamic shared memory bytes, CTAs per launch, and
        whether the angular tables store conjugate-paired polarisations once."""
        self._check()
        out = (ctypes.c_int * 14)()
        if self._lib.ctpwa_launch_shape(self._h, out) != 0:
            raise RuntimeError(_lib.error(self._h))
        keys = ("block", "min_ctas_per_sm", "stage", "acc_smem", "dyn_smem", "grid", "pol_paired")
        return {pr: dict(zip(keys, out[7 * i:7 * i + 7])) for i, pr in enumerate(("fp64", "mixed"))}

    def setKernelTiming(self, slots: int):
        """Record CUDA events around each fused-kernel launch (ring of `slots`; 0 = off)."""
        self._check()
        if self._lib.ctpwa_kernel_timing(self._h, int(slots)) != 0:
            raise RuntimeError(_lib.error(self._h))

    def kernelTimes(self, cap: int = 1 << 16):
        """Durations (ms) of the most recent fused-kernel launches, oldest first."""
        self._check()
        buf = (ctypes.c_float * cap)()
        n = self._lib.ctpwa_kernel_times(self._h, buf, cap)
        if n < 0:
            raise RuntimeError(_lib.error(self._h))
        return [buf[i] for i in range(n)]

    def lastParts(self):
        """[data_nll, bkg_nll, sum_phsp_intensity, W_data, W_bkg, n_phsp] of the last evaluation."""
        self._check()
        import numpy as np

        out = np.zeros(6)
        stream = torch.cuda.current_stream(self._device).cuda_stream
        rc = self._lib.ctpwa_last_parts(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError(_lib.error(self._h))
        return out

    def getCovariance(self, params: torch.Tensor, free=None, hessian: torch.Tensor = None) -> torch.Tensor:
        """Covariance of the fitted parameters: the inverse of the FP64 Hessian
        over the free parameters, formed and inverted on the device (the
        reference's fit driver inverts getHessian, example/fit.py:213,333).
        free: boolean mask over the parameters (default: all but the fixed
        first coupling, example/fit.py:48). float64 CUDA [nP, nP], zero in the
        rows and columns of fixed parameters."""
        p = self._check_params(params)
        nP, n = self.getNParams(), self.getNVector()
        if free is None:
            mask = torch.ones(nP, dtype=torch.bool)
            mask[0] = mask[n] = False
        else:
            mask = torch.as_tensor(free, dtype=torch.bool).reshape(-1)
            if mask.numel() != nP:
                raise RuntimeError(f"free mask must have {nP} entries")
        H = hessian if hessian is not None else self.getHessian(p)
        idx = torch.nonzero(mask).reshape(-1).to(p.device)
        Hf = H.to(device=p.device, dtype=torch.float64).index_select(0, idx).index_select(1, idx)
        C = torch.zeros((nP, nP), dtype=torch.float64, device=p.device)
        C[idx.unsqueeze(1), idx.unsqueeze(0)] = spd_inverse(Hf)
        return C

    def getHessian(self, params: torch.Tensor, method: str = "exact", rel_step: float = 1e-5) -> torch.Tensor:
        """Hessian [(2nV+nT), (2nV+nT)] (float64, CUDA), grouped [Re p, Im p, theta].

        method "exact" (default): forward-mode (dual-number) derivatives of the
        FP64 device gradient pass along every unit direction, symmetrised.
        method "fd": central differences of the exact FP64 device gradient with
        steps rel_step * max(|p_i|, 1e-2).
        method "gram": the coupling block from tensor-core Gram sums over the
        samples (FP32 amplitudes, split-BF16 products, FP64 assembly; ~1e-6
        relative to "exact"), the resonance-parameter rows exact; models with
        (npol + 1) * 2 * nA <= 128."""
        p = self._check_params(params)
        H = torch.empty((self._np, self._np), dtype=torch.float64, device=p.device)
        stream = torch.cuda.current_stream(p.device).cuda_stream
        if method == "exact":
            rc = self._lib.ctpwa_hessian_exact(self._h, p.data_ptr(), H.data_ptr(), ctypes.c_void_p(stream))
        elif method == "fd":
            rc = self._lib.ctpwa_hessian(self._h, p.data_ptr(), H.data_ptr(), float(rel_step), ctypes.c_void_p(stream))
        elif method == "gram":
            rc = self._lib.ctpwa_hessian_gram(self._h, p.data_ptr(), H.data_ptr(), ctypes.c_void_p(stream))
        else:
            raise ValueError('method must be "exact", "fd" or "gram"')
        if rc != 0:
            raise RuntimeError(_lib.error(self._h))
        return H

    def _check_dirs(self, p: torch.Tensor, dirs: torch.Tensor) -> torch.Tensor:
        if dirs.dim() == 1:
            dirs = dirs.unsqueeze(0)
        if dirs.dim() != 2 or dirs.shape[1] != self._np:
            raise ValueError(f"directions must have shape [ndir, {self._np}]")
        return dirs.to(device=p.device, dtype=torch.float64).contiguous()

    def getHessianVectorProduct(self, params: torch.Tensor, dirs: torch.Tensor) -> torch.Tensor:
        """Exact H(params) u for each row u of dirs ([ndir, nP] or [nP]);
        float64 CUDA [ndir, nP]."""
        p = self._check_params(params)
        d = self._check_dirs(p, dirs)
        out = torch.empty_like(d)
        stream = torch.cuda.current_stream(p.device).cuda_stream
        if self._lib.ctpwa_hvp(self._h, p.data_ptr(), d.data_ptr(), d.shape[0], out.data_ptr(),
                               ctypes.c_void_p(stream)) != 0:
            raise RuntimeError(_lib.error(self._h))
        return out

    def getGram(self, params: torch.Tensor) -> torch.Tensor:
        """Phase-space normalisation matrix M_ab = (1/W) sum_e w_e sum_pol
        A_a conj(A_b) at params (the reference's phase-space CGEMM matrix),
        on the tensor cores from the mixed-form amplitudes: complex128 CUDA
        [nA, nA]."""
        p = self._check_params(params)
        nA = self._nA if getattr(self, "_nA", None) else len(self.getAmplitudeNames())
        self._nA = nA
        out = torch.empty((nA, nA, 2), dtype=torch.float64, device=p.device)
        stream = torch.cuda.current_stream(p.device).cuda_stream
        if self._lib.ctpwa_gram(self._h, p.data_ptr(), out.data_ptr(), ctypes.c_void_p(stream)) != 0:
            raise RuntimeError(_lib.error(self._h))
        return torch.view_as_complex(out)

    def getShardHvpSums(self, params: torch.Tensor, dirs: torch.Tensor) -> torch.Tensor:
        """This shard's tangent sums for the directions (float64 CUDA, to be
        summed over shards and passed to finalizeShardHvp)."""
        p = self._check_params(params)
        d = self._check_dirs(p, dirs)
        out = torch.empty(self._lib.ctpwa_hvp_sums_size(self._h, d.shape[0]), dtype=torch.float64, device=p.device)
        stream = torch.cuda.current_stream(p.device).cuda_stream
        if self._lib.ctpwa_shard_hvp_sums(self._h, p.data_ptr(), d.data_ptr(), d.shape[0], out.data_ptr(),
                                          ctypes.c_void_p(stream)) != 0:
            raise RuntimeError(_lib.error(self._h))
        return out

    def finalizeShardHvp(self, params: torch.Tensor, dirs: torch.Tensor, sums: torch.Tensor,
                         hvp_sums: torch.Tensor) -> torch.Tensor:
        """Rows H u of the union of the shards from the summed FP64 shard sums
        (getShardSums(params, "fp64")) and the summed tangent sums."""
        p = self._check_params(params)
        d = self._check_dirs(p, dirs)
        if sums.dtype != torch.float64 or not sums.is_cuda or sums.numel() != self._lib.ctpwa_sums_size(self._h):
            raise RuntimeError("sums must be the float64 CUDA buffer of getShardSums")
        if (hvp_sums.dtype != torch.float64 or not hvp_sums.is_cuda
                or hvp_sums.numel() != self._lib.ctpwa_hvp_sums_size(self._h, d.shape[0])):
            raise RuntimeError("hvp_sums must be the float64 CUDA buffer of getShardHvpSums")
        sums, hvp_sums = sums.contiguous(), hvp_sums.contiguous()
        out = torch.empty_like(d)
        stream = torch.cuda.current_stream(p.device).cuda_stream
        if self._lib.ctpwa_finalize_hvp(self._h, p.data_ptr(), d.data_ptr(), d.shape[0], sums.data_ptr(),
                                        hvp_sums.data_ptr(), out.data_ptr(), ctypes.c_void_p(stream)) != 0:
            raise RuntimeError(_lib.error(self._h))
        return out
