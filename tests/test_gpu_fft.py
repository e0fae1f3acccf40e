"""FFT Poisson parity: the in-house FFT path against numpy.fft restatements.

Periodic mode follows Compute_hartree_fft (qmtools/qmtools.py:2578-2639,
kernel_fft.cu:23-107); padded mode is the Hockney free-space solve.
"""
import numpy as np
import pytest

import qmtools
from qmtools import synthetic as syn
from oracle import poisson as op
from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 2e-5   # FP32 transforms against FP64 numpy.fft


@pytest.fixture(scope="module")
def c0(basis):
    sm = syn.config_molecule("c0")
    return sm, sm.molecule(basis, qmtools.Molecule)


def _density(mol, shape, step, centre):
    n = np.array(shape)
    g = qmtools.Grid((1,) + tuple(shape), step / qmtools.ANG2BOR, list(centre - n * step / 2))
    return qmtools.QMTools.Compute_density(g, mol, precision="fp32")


# 256- and 128-point lines (one axis each) take the register kernels in every pass mode; other
# lengths the shared-memory one
@pytest.mark.parametrize("shape", [(32, 32, 32), (24, 40, 56), (136, 16, 24), (48, 8, 88),
                                   (256, 16, 8), (16, 256, 8), (8, 16, 256),
                                   (128, 16, 8), (16, 128, 8), (8, 16, 128)])
def test_periodic_matches_numpy(c0, shape):
    sm, mol = c0
    q = _density(mol, shape, 0.35, np.asarray(sm.coords_bohr).mean(axis=0))
    got = qmtools.QMTools.Compute_hartree_fft(q, mol, sigma=0.2, cutoff=6)
    nx, ny, nz, h, ox, oy, oz = q._geom()
    ref = op.fft_poisson_periodic(q.qube.ravel(), (nx, ny, nz), h, (ox, oy, oz), mol.coords, mol.types, 0.2, 6)
    assert got.shape == (nx, ny, nz)
    assert rel_l2(got, ref) < TOL


@pytest.mark.parametrize("shape", [(32, 32, 32), (24, 16, 40), (128, 8, 16), (8, 128, 16), (16, 8, 128),
                                   (64, 8, 16), (8, 64, 16), (16, 8, 64)])
def test_hockney_matches_numpy(c0, shape):
    sm, mol = c0
    q = _density(mol, shape, 0.4, np.asarray(sm.coords_bohr).mean(axis=0))
    got = qmtools.QMTools.Compute_hartree_fft(q, mol, sigma=0.2, cutoff=6, padded=True)
    nx, ny, nz, h, ox, oy, oz = q._geom()
    ref = op.hockney_poisson(q.qube.ravel(), (nx, ny, nz), h, (ox, oy, oz), mol.coords, mol.types, 0.2, 6)
    assert rel_l2(got, ref) < TOL


def test_hockney_is_deterministic(c0):
    sm, mol = c0
    q = _density(mol, (32, 32, 32), 0.4, np.asarray(sm.coords_bohr).mean(axis=0))
    a = qmtools.QMTools.Compute_hartree_fft(q, mol, padded=True)
    b = qmtools.QMTools.Compute_hartree_fft(q, mol, padded=True)
    assert np.array_equal(a, b)
