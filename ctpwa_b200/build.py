"""In-tree build of libctpwa_b200.so (host C++ + sm_100a CUDA, NVRTC at run time).

Usage: python -m ctpwa_b200.build [--force]
The shared library is written next to this file; the kernel sources under
csrc/kernels/ are read by the library at run time and compiled by NVRTC for
sm_100a per physics model.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libctpwa_b200.so"
BUILD = PKG / "_build"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA / "bin" / "nvcc")
HOSTCXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

HOST_SRCS = ["yaml_lite.cpp", "config.cpp", "model.cpp", "dataio.cpp", "exprdag.cpp", "lineshape_lang.cpp", "codegen.cpp", "fit.cpp",
             "capi.cpp"]
CUDA_SRCS = ["engine.cu", "toymc.cu", "linalg.cu"]


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    return r


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "ctpwa_b200.h"]
    objs = []
    for s in HOST_SRCS:
        src = CSRC / s
        obj = BUILD / (s + ".o")
        if force or _newer(obj, [src] + headers):
            _run([HOSTCXX, "-O2", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function",
                  f"-I{CUDA / 'include'}", "-c", str(src), "-o", str(obj)])
        objs.append(obj)
    for s in CUDA_SRCS:
        src = CSRC / s
        obj = BUILD / (s + ".o")
        if force or _newer(obj, [src] + headers):
            r = _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-ccbin", HOSTCXX,
                      "-Xcompiler", "-fPIC", "-Xptxas", "-v", "-c", str(src), "-o", str(obj)])
            if verbose:
                sys.stderr.write(r.stderr)
        objs.append(obj)
    if force or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-ccbin", HOSTCXX, "-o", str(LIB), *map(str, objs),
              f"-L{CUDA / 'lib64'}", "-lcudart", "-lnvrtc", "-ldl",
              "-Xlinker", f"-rpath,{CUDA / 'lib64'}"])
    return LIB


def precompile_workloads() -> None:
    """Fill the package kernel cache with the fused kernels of the bundled
    benchmark models (NVRTC for sm_100a, no GPU needed)."""
    import tempfile

    from . import precompile, workloads

    with tempfile.TemporaryDirectory(prefix="ctpwa_pre_") as d:
        for name in workloads.SIZES:
            cfg = Path(d) / f"{name}.yml"
            cfg.write_text(workloads.config_text(name, f"{d}/phsp.npy", f"{d}/data.npy", f"{d}/bkg.npy", 0.5))
            precompile(str(cfg))


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
