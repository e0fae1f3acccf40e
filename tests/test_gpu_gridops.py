"""Grid utilities, nuclear seed and Vne fields against the oracle."""
import numpy as np
import pytest

import qmtools
from qmtools import synthetic as syn
from oracle import gridops as og
from oracle import poisson as op
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c0(basis):
    sm = syn.config_molecule("c0")
    return sm, sm.molecule(basis, qmtools.Molecule)


def _grid(sm, n, step):
    c = np.asarray(sm.coords_bohr).mean(axis=0)
    return qmtools.Grid((1, n, n, n), step / qmtools.ANG2BOR, list(c - n * step / 2))


def test_qtot_qscale_qdiff():
    rng = np.random.default_rng(5)
    g1 = qmtools.Grid((1, 24, 16, 8), 0.1)
    g2 = qmtools.Grid((1, 24, 16, 8), 0.1)
    a = rng.uniform(0.1, 2.0, size=g1.qube.shape).astype(np.float32)
    b = rng.uniform(0.1, 2.0, size=g1.qube.shape).astype(np.float32)
    g1.LoadFromNPY(a)
    g2.LoadFromNPY(b)
    T = qmtools.QMTools
    assert abs(T.Compute_qtot(g1) - og.qtot(a)) < 1e-9 * og.qtot(a)
    assert abs(T.Compute_qdiff(g1, g2) - og.qdiff(a, b)) < 1e-9 * og.qdiff(a, b)
    assert abs(T.Compute_qdiff(g1, g2, rel=True) - og.qdiff(a, b, rel=True)) < 1e-5 * og.qdiff(a, b, rel=True)
    T.Compute_qscale(g1, 0.5, copyBack=True)
    assert np.array_equal(g1.qube, (a * np.float32(0.5)).astype(np.float32))
    e = T.Compute_errors(g1, g2)
    d = g1.qube.astype(np.float64) - b
    assert abs(e["max_abs"] - np.abs(d).max()) < 1e-12
    assert abs(e["rel_l2"] - np.linalg.norm(d) / np.linalg.norm(b.astype(np.float64))) < 1e-12


def test_density_seed_bit_exact(c0):
    sm, mol = c0
    g = _grid(sm, 40, 0.25)
    got = qmtools.QMTools.Compute_qseed(g, mol).qube.ravel()
    ref = op.density_seed(g.space_shape(), g.step, g._geom()[4:], mol.coords, mol.types)
    assert np.array_equal(got, ref)
    assert abs(got.sum(dtype=np.float64) - mol.qtot) < 1e-4


def test_vne_point(c0):
    sm, mol = c0
    g = _grid(sm, 24, 0.5)
    got = qmtools.QMTools.Compute_VNe_point(g, mol).qube.ravel()
    ref = og.vne_centres(g.space_shape(), g.step, g._geom()[4:], mol.coords, mol.types)
    assert rel_l2(got, ref) < 1e-6


def test_vne_classic(c0):
    sm, mol = c0
    g = _grid(sm, 16, 0.5)
    got = qmtools.QMTools.Compute_VNe_classic(g, mol, divisions=3).qube.ravel()
    ref = og.vne_classic(g.space_shape(), g.step, g._geom()[4:], mol.coords, mol.types, divisions=3)
    assert rel_l2(got, ref) < 1e-5


def test_vne_pseudo_field(c0):
    sm, mol = c0
    g = _grid(sm, 16, 0.5)
    got = qmtools.QMTools.Compute_VNe(g, mol, adsorb=0.05, diff=0.02, tolerance=1e-9, maxiters=6)
    ref, it = og.vne_pseudo(g.space_shape(), g.step, g._geom()[4:], mol.coords, mol.types, ads=0.05, dif=0.02,
                            tolerance=1e-9, maxiters=6)
    assert got.iterations == it
    assert rel_l2(got.qube.ravel(), ref) < 1e-5
