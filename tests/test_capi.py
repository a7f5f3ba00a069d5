"""The C ABI library loads and exports every symbol include/ctpwa_b200.h declares."""
import ctypes
import os
import re

import ctpwa_b200
from ctpwa_b200 import _lib, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "ctpwa_b200.h")).read()
    return sorted(set(re.findall(r"\b(ctpwa_[a-z_0-9]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    syms = declared_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(lib, s), s


def test_binding_covers_header():
    assert set(declared_symbols()) == set(_lib.SIGNATURES)


def test_version_and_errors(tmp_path):
    assert ctpwa_b200.version().startswith("ctpwa_b200")
    lib = _lib.load()
    st = ctypes.c_int(0)
    err = ctypes.create_string_buffer(256)
    h = lib.ctpwa_create(str(tmp_path / "none.yml").encode(), 0, ctypes.byref(st), err, 256)
    assert not h and st.value == -1 and b"not initialized" in err.value
    assert b"not initialized" in lib.ctpwa_last_error(None)


def test_precompile_without_gpu(tmp_path):
    p = tmp_path / "c.yml"
    p.write_text(workloads.config_text("pipi_rho", "p.npy", "d.npy"))
    assert ctpwa_b200.precompile(str(p)) >= 0.0


def test_null_handle_arguments_are_rejected():
    """Entry points given no handle or no buffers return CTPWA_ERR_ARG (or 0
    for the queries) without touching a device."""
    lib = _lib.load()
    ERR_ARG = -3  # CTPWA_ERR_ARG
    dp = ctypes.c_void_p(0)
    assert lib.ctpwa_norm_cache_valid(None) == 0
    assert lib.ctpwa_norm_cache_clear(None) == ERR_ARG
    assert lib.ctpwa_norm_cache_build(None, dp, None, None) == ERR_ARG
    assert lib.ctpwa_nll_grad_cached(None, dp, dp, dp, 0, None) == ERR_ARG
    assert lib.ctpwa_nll_grad(None, dp, dp, dp, 0, None) == ERR_ARG
