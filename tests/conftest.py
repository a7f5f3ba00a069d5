import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the device path")


def cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def reference_root():
    """The reference source tree, when this machine has it: the
    CTPWA_REFERENCE_ROOT environment variable, else the tree the oracle's
    reference-math library was built from (oracle/_ref/ref_root.txt). None
    where neither names an existing directory (the GPU box has no copy)."""
    cand = os.environ.get("CTPWA_REFERENCE_ROOT")
    if not cand:
        rec = os.path.join(ROOT, "oracle", "_ref", "ref_root.txt")
        if os.path.exists(rec):
            cand = open(rec).read().strip()
    return cand if cand and os.path.isdir(cand) else None
