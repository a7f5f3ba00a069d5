"""ORACLE BUILD RECIPE — test infrastructure, not product code.

Builds the reference's own CUDA extension (the `ctpwa` pybind11 module) from
its sources where they lie, unmodified, for sm_100 (B200), in the two
precisions it supports: `oracle/_ref/cuda_f64/ctpwa.so` (complex<double>,
the reference built with CTPWA_DOUBLE_COMPLEX=1) and
`oracle/_ref/cuda_f32/ctpwa.so` (its default complex<float> build).

The reference's setup.py links yaml-cpp and ROOT, neither of which exists
here or on the GPU box, and reads ROOT's location from root-config; this
recipe compiles the same source list with the same nvcc options, and stands
in for the two libraries with oracle/refcuda/shim (yaml-cpp: the node API
over trees composed by PyYAML; ROOT: declarations whose file IO fails as a
missing file does). The likelihood path (config.yml, .dat samples, getNLL,
getHessian) uses neither library.

Usage: python -m oracle.refcuda.build [--ref REF_ROOT] [--only f64|f32]
The reference root defaults to CTPWA_REFERENCE_ROOT, else /root/reference.
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ORACLE = HERE.parent
OUT = ORACLE / "_ref"

# src/ list of the reference's setup.py:128-141
SOURCES = ["src/main.cu", "src/Amplitude.cu", "src/ComputeHessian.cu", "src/AmpGen.cu", "src/ComputeNLL.cu",
           "src/ComputeResults.cu", "src/ComputeBF.cu", "src/Figure.cu", "src/Parameters.cu", "src/CustomExpr.cu",
           "src/JITCustom.cu"]


def build_one(ref: Path, precision: str, jobs: int) -> Path:
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    # the system compilers: the extension must use the process's shared
    # libstdc++ (a statically linked copy breaks iostreams and exceptions
    # across the pybind11 boundary)
    os.environ["CC"] = os.environ.get("CTPWA_REF_CC", "/usr/bin/gcc")
    os.environ["CXX"] = os.environ.get("CTPWA_REF_CXX", "/usr/bin/g++")
    os.environ.setdefault("MAX_JOBS", str(jobs))
    from setuptools import setup
    from torch.utils.cpp_extension import BuildExtension, CUDAExtension

    cuda = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
    dest = OUT / f"cuda_{precision}"
    dest.mkdir(parents=True, exist_ok=True)
    # a fixed build folder outside the repository, so that ninja rebuilds only
    # what changed; setuptools wants sources relative to the working
    # directory: the reference tree and the shim are linked in (read only)
    tmp = Path(tempfile.gettempdir()) / f"ctpwa_refcuda_{precision}"
    tmp.mkdir(exist_ok=True)
    for name, target in (("ref", ref), ("shim", HERE / "shim")):
        link = tmp / name
        if link.is_symlink() and Path(os.readlink(link)) != Path(target):
            link.unlink()
        if not link.exists():
            os.symlink(target, link)
    nvcc = ["-rdc=true", "--expt-relaxed-constexpr", "-std=c++17", "--extended-lambda"]
    if precision == "f64":
        nvcc.append("-DCTPWA_DOUBLE_COMPLEX")
    ext = CUDAExtension(
        name="ctpwa",
        sources=[f"ref/{s}" for s in SOURCES] + ["shim/yaml_shim.cpp"],
        include_dirs=[str(tmp / "shim"), str(ref / "include"), str(cuda / "include")],
        library_dirs=[str(cuda / "lib64"), str(cuda / "lib64" / "stubs")],
        libraries=["cudart", "cublas", "nvrtc", "cuda"],
        extra_compile_args={"cxx": ["-fPIC", "-std=c++17", "-w"], "nvcc": nvcc + ["-w"], "nvcc_dlink": ["-dlink"]},
        extra_link_args=["-Wl,--no-as-needed"],
    )
    cwd = os.getcwd()
    try:
        os.chdir(tmp)
        setup(name="ctpwa_reference_build", ext_modules=[ext],
              cmdclass={"build_ext": BuildExtension.with_options(use_ninja=True, no_python_abi_suffix=True)},
              script_args=["-q", "build_ext", "--build-lib", str(dest), "--build-temp", str(tmp / "build")])
    finally:
        os.chdir(cwd)
    so = dest / "ctpwa.so"
    if not so.exists():
        raise RuntimeError(f"reference build produced no {so}")
    (dest / "ref_root.txt").write_text(str(ref) + "\n")
    return so


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("CTPWA_REFERENCE_ROOT", "/root/reference"))
    ap.add_argument("--only", choices=["f64", "f32"])
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    a = ap.parse_args(argv)
    ref = Path(a.ref)
    if not (ref / "src" / "main.cu").exists():
        sys.exit(f"reference tree not found at {ref}")
    for prec in ([a.only] if a.only else ["f64", "f32"]):
        print(build_one(ref, prec, a.jobs))


if __name__ == "__main__":
    main()
