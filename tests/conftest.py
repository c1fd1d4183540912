"""Shared pytest configuration.

Markers
  gpu  -- needs a CUDA device (B200); run with `pytest -m gpu`.  Everything
          else runs on CPU (`pytest -m "not gpu"`).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
# The reference's sources: $REF, else the oracle build recipe's default.  The
# tests that read them skip where they are absent (as on a GPU box).
from oracle import reference_root  # noqa: E402

REF = reference_root()
REF_MB = os.path.join(REF, "Release_MBFPA_CPU_human")
REF_FBP = os.path.join(REF, "Release_FBP_CPU")

# Tolerances stated by the task: noise-free sinograms within 1e-5 relative
# per element; FBP images within 1e-4 of max|ref| per pixel and 1e-4 in
# relative L2 (the image crosses zero).
SINO_RTOL = 1e-5
FBP_ATOL_REL = 1e-4
FBP_L2_REL = 1e-4


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu)")


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def have_reference_sources():
    return os.path.isdir(REF_MB) and os.path.isdir(REF_FBP)


def max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.abs(b)))


def fbp_errors(img, ref):
    img = np.asarray(img, np.float64)
    ref = np.asarray(ref, np.float64)
    scale = np.max(np.abs(ref))
    return float(np.max(np.abs(img - ref)) / scale), float(np.linalg.norm(img - ref) / np.linalg.norm(ref))


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return 0
