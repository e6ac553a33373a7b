"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
PKG = REPO / "berkeleygw-kernels-cpp_b200"
for p in (PKG, REPO, REPO / "tests" / "golden"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

# Parity bar of the plain FP64 form against the reference / the oracle.
FP64_RTOL = 1e-12
# Bar of the mixed-precision GPP band loop (hoisted FP64 expansion terms,
# FP32 remainder quotients) against the FP64 oracle: 1e-9 relative.
MIXED_RTOL = 1e-9


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def rel_err(got, ref) -> float:
    """max |got - ref| / max |ref| over a (complex) array; absolute if ref is 0."""
    got = np.atleast_1d(np.asarray(got, dtype=np.complex128))
    ref = np.atleast_1d(np.asarray(ref, dtype=np.complex128))
    assert got.shape == ref.shape, (got.shape, ref.shape)
    scale = float(np.max(np.abs(ref))) if ref.size else 0.0
    diff = float(np.max(np.abs(got - ref))) if ref.size else 0.0
    return diff / scale if scale > 0 else diff


def l2c(lst) -> np.ndarray:
    return np.array([complex(a, b) for a, b in lst], dtype=np.complex128)


@pytest.fixture(scope="session")
def golden():
    return json.loads((REPO / "tests" / "golden" / "golden.json").read_text())


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def bgw():
    import bgwsigma
    bgwsigma.load()
    return bgwsigma


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test needs a CUDA device")
    return torch.device("cuda:0")
