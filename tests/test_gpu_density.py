"""Density parity: the CUDA path (every precision) against the FP64 oracle.

The oracle restates `gpu_densityqube_shmem_subgrid` (kernel_density.cu:34-155) and the
qtot rescale of `Compute_density` (qmtools/qmtools.py:2419-2424).
"""
import numpy as np
import pytest

import qmtools
from qmtools import synthetic as syn
from oracle import density as od
from conftest import rel_l2

pytestmark = pytest.mark.gpu

# rel-L2 tolerance of the unscaled grid against the FP64 oracle, per precision (the grid is
# stored in float32, so even the FP64 path carries ~3e-8 of output rounding)
TOL = {"fp64": 1e-7, "fp32": 1e-6, "fp16x3": 1e-6, "tf32x3": 2e-6, "bf16x3": 1e-4,
       "tf32": 5e-3, "bf16": 5e-2}


def _small_grid(sm, n, step):
    c = np.asarray(sm.coords_bohr).mean(axis=0)
    o = c - n * step / 2
    return qmtools.Grid((1, n, n, n), step / qmtools.ANG2BOR, list(o))


def _oracle(grid, mol, subgrid=1):
    nx, ny, nz, h, ox, oy, oz = grid._geom()
    return od.density_qube_unscaled((nx, ny, nz), np.float32(h), (ox, oy, oz), mol.coords, mol.ALMOs,
                                    mol.basisset.alphas, mol.basisset.coeffs, mol.dm, subgrid)


@pytest.fixture(scope="module")
def c0(basis):
    sm = syn.config_molecule("c0")
    return sm, sm.molecule(basis, qmtools.Molecule)


@pytest.fixture(scope="module")
def c1(basis):
    sm = syn.config_molecule("c1")
    return sm, sm.molecule(basis, qmtools.Molecule)


@pytest.mark.parametrize("prec", list(TOL))
def test_density_c0_all_precisions(c0, prec):
    sm, mol = c0
    g = _small_grid(sm, 32, 0.4)
    ref = _oracle(g, mol)
    out = qmtools.QMTools.Compute_density(g, mol, precision=prec, rescale=False)
    got = out.qube.ravel()
    err = rel_l2(got, ref)
    assert err <= TOL[prec], f"{prec}: rel-L2 {err:.3e}"
    assert abs(out.qsum - ref.sum()) <= max(10 * TOL[prec], 1e-9) * abs(ref.sum())


@pytest.mark.parametrize("prec", ["fp32", "fp16x3", "tf32x3", "bf16x3"])
def test_density_two_panels(c1, prec):
    """N = 294 needs two output panels in the tensor-core kernel."""
    sm, mol = c1
    g = _small_grid(sm, 24, 0.8)
    ref = _oracle(g, mol)
    out = qmtools.QMTools.Compute_density(g, mol, precision=prec, rescale=False)
    assert rel_l2(out.qube.ravel(), ref) <= TOL[prec]


@pytest.mark.parametrize("prec", ["fp32", "fp16x3"])
def test_density_subgrid2(c0, prec):
    sm, mol = c0
    g = _small_grid(sm, 16, 0.6)
    ref = _oracle(g, mol, subgrid=2)
    out = qmtools.QMTools.Compute_density(g, mol, subgrid=2, precision=prec, rescale=False)
    assert rel_l2(out.qube.ravel(), ref) <= TOL[prec]


@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16x3"])
def test_density_sample_molecule(sample_molecule, prec):
    """Real molecule with Br/Cl (d shells with 5 primitives) and a CCSD density matrix."""
    mol = sample_molecule
    g = qmtools.Grid.DensityGrid(mol, 0.35, 1.0)
    ref = _oracle(g, mol)
    out = qmtools.QMTools.Compute_density(g, mol, precision=prec, rescale=False)
    assert rel_l2(out.qube.ravel(), ref) <= TOL[prec]


def test_density_rescale_matches_reference_convention(c0):
    """After Compute_density the grid sums to the nuclear charge (qmtools/qmtools.py:2419-2424)."""
    sm, mol = c0
    g = _small_grid(sm, 32, 0.4)
    q, _, _ = od.compute_density(g.space_shape(), np.float32(g.step), g._geom()[4:], mol.coords, mol.types,
                                 mol.ALMOs, mol.basisset.alphas, mol.basisset.coeffs, mol.dm)
    out = qmtools.QMTools.Compute_density(g, mol, precision="fp32")
    assert abs(float(np.sum(out.qube, dtype=np.float64)) - float(mol.qtot)) < 1e-3
    assert rel_l2(out.qube.ravel(), q) <= 2e-6


def test_trace_ps(c0):
    from oracle import integrals as oi
    sm, mol = c0
    S = oi.overlap_matrix(mol.coords, mol.ALMOs, mol.basisset.alphas, mol.basisset.coeffs)
    P = oi.sym_lower(mol.dm)
    assert abs(mol.trace_ps() - float(np.sum(P * S))) < 1e-10


def test_density_deterministic(c1):
    sm, mol = c1
    g = _small_grid(sm, 24, 0.8)
    a = qmtools.QMTools.Compute_density(g, mol, precision="fp16x3")
    b = qmtools.QMTools.Compute_density(g, mol, precision="fp16x3")
    assert np.array_equal(a.qube, b.qube)
    assert a.qsum == b.qsum


@pytest.fixture(params=[1, 2, 3], ids=["staged", "fused", "fused_tri"])
def density_path(request):
    """Run a test once through each tensor-core implementation, then restore automatic choice."""
    from qmtools import _native as N
    N.call("qmt_set_density_path", request.param)
    yield request.param
    N.call("qmt_set_density_path", 0)


@pytest.mark.parametrize("prec", ["fp16x3", "bf16x3", "bf16"])
def test_density_paths_agree_with_oracle(c1, density_path, prec):
    """Staged (HBM) and fused (shared-memory, upper-triangular) tensor-core paths, N = 294."""
    sm, mol = c1
    g = _small_grid(sm, 24, 0.8)
    ref = _oracle(g, mol)
    out = qmtools.QMTools.Compute_density(g, mol, precision=prec, rescale=False)
    # the triangular variant accumulates larger partial sums in FP32 (about 2x the error)
    tol = TOL[prec] * (3 if density_path == 3 else 1)
    assert rel_l2(out.qube.ravel(), ref) <= tol


@pytest.mark.parametrize("sub", [1, 2, 3])
def test_fused_path_subgrids_and_small_basis(c0, density_path, sub):
    """N = 58 (one 64-wide K block), partial last tile, sub-point averaging."""
    sm, mol = c0
    g = _small_grid(sm, 16 if sub > 1 else 24, 0.6)
    ref = _oracle(g, mol, subgrid=sub)
    out = qmtools.QMTools.Compute_density(g, mol, subgrid=sub, precision="fp16x3", rescale=False)
    assert rel_l2(out.qube.ravel(), ref) <= TOL["fp16x3"] * (3 if density_path == 3 else 1)
