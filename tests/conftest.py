"""Shared test set-up: import paths, the `gpu` marker and common fixtures."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "qmtools-pycuda_b200"))
sys.path.insert(0, str(ROOT))

import qmtools  # noqa: E402

qmtools.set_verbose(False)

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built CUDA library")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def basis():
    return qmtools.BasisSet(qmtools.BASIS_CCPVDZ)


@pytest.fixture(scope="session")
def sample_molecule(basis):
    """The real molecule shipped with the reference (Br, 2 Cl, 6 C, 3 H; N = 162; CCSD DM)."""
    d = GOLDEN / "molecule_29766_0"
    return qmtools.Molecule(str(d / "GEOM-B3LYP.xyz"), str(d / "D-CCSD.npy"), basis)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
