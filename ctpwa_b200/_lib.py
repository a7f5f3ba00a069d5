"""ctypes binding of libctpwa_b200.so (the C ABI declared in include/ctpwa_b200.h)."""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("CTPWA_B200_LIB", _PKG / "libctpwa_b200.so"))

_c_double_p = ctypes.POINTER(ctypes.c_double)

# name: (restype, argtypes)
SIGNATURES = {
    "ctpwa_create": (ctypes.c_void_p, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                       ctypes.c_char_p, ctypes.c_size_t]),
    "ctpwa_create_from_device": (ctypes.c_void_p, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                                   ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_void_p),
                                                   ctypes.POINTER(ctypes.c_int), ctypes.c_char_p, ctypes.c_size_t]),
    "ctpwa_create_from_device_flags": (ctypes.c_void_p, [ctypes.c_char_p, ctypes.c_int,
                                                         ctypes.POINTER(ctypes.c_void_p),
                                                         ctypes.POINTER(ctypes.c_longlong),
                                                         ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                                         ctypes.POINTER(ctypes.c_int), ctypes.c_char_p,
                                                         ctypes.c_size_t]),
    "ctpwa_create_shard": (ctypes.c_void_p, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_int), ctypes.c_char_p, ctypes.c_size_t]),
    "ctpwa_destroy": (None, [ctypes.c_void_p]),
    "ctpwa_hessian": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                     ctypes.c_void_p]),
    "ctpwa_hessian_exact": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "ctpwa_hessian_gram": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "ctpwa_gram_shape": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "ctpwa_gram": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "ctpwa_norm_cache_build": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                              ctypes.c_void_p]),
    "ctpwa_norm_cache_clear": (ctypes.c_int, [ctypes.c_void_p]),
    "ctpwa_norm_cache_valid": (ctypes.c_int, [ctypes.c_void_p]),
    "ctpwa_nll_grad_cached": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_int, ctypes.c_void_p]),
    "ctpwa_batch_create": (ctypes.c_void_p, [ctypes.c_int]),
    "ctpwa_batch_destroy": (None, [ctypes.c_void_p]),
    "ctpwa_nll_grad_multi": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "ctpwa_batch_join": (ctypes.c_int, [ctypes.c_void_p]),
    "ctpwa_batch_leave": (ctypes.c_int, [ctypes.c_void_p]),
    "ctpwa_batch_eval_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_int]),
    "ctpwa_batch_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "ctpwa_fit_batched": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]),
    "ctpwa_spd_inverse": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    "ctpwa_hvp": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                 ctypes.c_void_p]),
    "ctpwa_hvp_sums_size": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "ctpwa_shard_hvp_sums": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                            ctypes.c_void_p, ctypes.c_void_p]),
    "ctpwa_finalize_hvp": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "ctpwa_n_blocks": (ctypes.c_int, [ctypes.c_void_p]),
    "ctpwa_partial_integrals": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                               ctypes.c_void_p]),
    "ctpwa_table_stride": (ctypes.c_longlong, [ctypes.c_void_p, ctypes.c_int]),
    "ctpwa_export_weights": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p]),
    "ctpwa_sums_size": (ctypes.c_int, [ctypes.c_void_p]),
    "ctpwa_shard_sums": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_void_p]),
    "ctpwa_finalize_sums": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p]),
    "ctpwa_n_vector": (ctypes.c_int, [ctypes.c_void_p]),
    "ctpwa_n_free_theta": (ctypes.c_int, [ctypes.c_void_p]),
    "ctpwa_n_params": (ctypes.c_int, [ctypes.c_void_p]),
    "ctpwa_param_names": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "ctpwa_free_res_params": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "ctpwa_nll_grad": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_int, ctypes.c_void_p]),
    "ctpwa_nll_grad_static": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_int, ctypes.c_void_p]),
    "ctpwa_nll_grad_host": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, _c_double_p, _c_double_p,
                                           ctypes.c_int, ctypes.c_void_p]),
    "ctpwa_intensity": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_void_p]),
    "ctpwa_last_parts": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, ctypes.c_void_p]),
    "ctpwa_n_events": (ctypes.c_longlong, [ctypes.c_void_p, ctypes.c_int]),
    "ctpwa_model_json": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "ctpwa_device_bytes": (ctypes.c_size_t, [ctypes.c_void_p]),
    "ctpwa_phase_space": (ctypes.c_int, [ctypes.c_double, ctypes.POINTER(ctypes.c_double), ctypes.c_longlong,
                                         ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_void_p]),
    "ctpwa_event_cache_layout": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "ctpwa_launch_shape": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "ctpwa_event_layout": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "ctpwa_kernel_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "ctpwa_kernel_times": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int]),
    "ctpwa_jit_seconds": (ctypes.c_double, [ctypes.c_void_p]),
    "ctpwa_setup_times": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "ctpwa_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "ctpwa_describe": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p,
                                      ctypes.c_size_t]),
    "ctpwa_precompile": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.c_char_p,
                                        ctypes.c_size_t]),
    "ctpwa_version": (ctypes.c_char_p, []),
    "ctpwa_fit": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, ctypes.POINTER(ctypes.c_ubyte), _c_double_p,
                                 _c_double_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_double, _c_double_p, ctypes.POINTER(ctypes.c_float), ctypes.c_void_p]),
    "ctpwa_fit_newton": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, ctypes.POINTER(ctypes.c_ubyte), _c_double_p,
                                        _c_double_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, _c_double_p, ctypes.c_void_p]),
    "ctpwa_minimize_box": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _c_double_p,
                                          ctypes.POINTER(ctypes.c_ubyte), _c_double_p, _c_double_p, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_double, ctypes.c_double, _c_double_p]),
    "ctpwa_minimize_box_newton": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                 _c_double_p, ctypes.POINTER(ctypes.c_ubyte), _c_double_p, _c_double_p,
                                                 ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                 _c_double_p]),
}

# host function for ctpwa_minimize_box: fn(x, &f, g, user) -> status
FG_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                         ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)
# host Hessian for ctpwa_minimize_box_newton: hfn(x, H, user) -> status
HESS_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                           ctypes.c_void_p)

_lib = None


def load():
    """Load the native library; raises ImportError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m ctpwa_b200.build` "
                          "(this package has no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def error(h) -> str:
    msg = load().ctpwa_last_error(h)
    return msg.decode("utf-8", "replace") if msg else ""


def read_string(fn, h) -> str:
    n = fn(h, None, 0)
    if n < 0:
        raise RuntimeError(error(h))
    buf = ctypes.create_string_buffer(n)
    fn(h, buf, n)
    return buf.value.decode("utf-8")
