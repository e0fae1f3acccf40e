"""Hartree routes against the oracle: analytic GTO potential, Jacobi, FP64 trace."""
import numpy as np
import pytest

import qmtools
from qmtools import synthetic as syn
from oracle import integrals as oi
from oracle import poisson as op
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c0(basis):
    sm = syn.config_molecule("c0")
    return sm, sm.molecule(basis, qmtools.Molecule)


def _grid(sm, n, step):
    c = np.asarray(sm.coords_bohr).mean(axis=0)
    return qmtools.Grid((1, n, n, n), step / qmtools.ANG2BOR, list(c - n * step / 2 + 0.013))


def test_gto_potential_corners(c0):
    """Compute_hartree at voxel corners vs the McMurchie-Davidson oracle (FP64 vs FP64)."""
    sm, mol = c0
    g = _grid(sm, 16, 0.7)
    qmtools.QMTools.Compute_hartree(g, mol)
    pts = oi.voxel_corners(g.space_shape(), g.step, g._geom()[4:])
    ref = oi.total_potential(pts, mol.coords, mol.types, mol.ALMOs, mol.basisset.alphas, mol.basisset.coeffs,
                             mol.dm)
    assert rel_l2(g.qube.ravel(), ref) < 1e-6


def test_gto_potential_sample_molecule_points(sample_molecule):
    """d shells, many primitives, real CCSD density matrix; arbitrary points."""
    import ctypes as C
    import torch
    mol = sample_molecule
    rng = np.random.default_rng(7)
    pts = (mol.coords.mean(axis=0) + rng.uniform(-6, 6, size=(300, 3))).astype(np.float32)
    pt = torch.from_numpy(pts.ravel()).cuda()
    out = torch.empty(300, dtype=torch.float32, device="cuda")
    from qmtools import _native as N
    N.call("qmt_hartree_gto_points", mol.handle, 300, C.c_void_p(pt.data_ptr()), C.c_void_p(out.data_ptr()),
           N.stream_handle())
    ref = oi.total_potential(pts, mol.coords, mol.types, mol.ALMOs, mol.basisset.alphas, mol.basisset.coeffs,
                             mol.dm)
    assert rel_l2(out.cpu().numpy(), ref) < 1e-6


def test_jacobi_reference_update(c0):
    """gpu_hartree_iteration semantics (kernel_hartree.cu:85-171), FP32 against an FP32 restatement."""
    import ctypes as C
    import torch
    from qmtools import _native as N
    sm, mol = c0
    g = _grid(sm, 24, 0.5)
    q = qmtools.QMTools.Compute_density(g, mol, precision="fp32")
    seed = qmtools.QMTools.Compute_qseed(g, mol)
    rho = (seed.qube.ravel() - q.qube.ravel()).astype(np.float32)
    nx, ny, nz, h, *_ = g._geom()
    r = torch.from_numpy(rho).cuda()
    v = torch.zeros_like(r)
    t = torch.zeros_like(r)
    sw = C.c_int()
    dl = C.c_double()
    N.call("qmt_jacobi", nx, ny, nz, h, C.c_void_p(r.data_ptr()), C.c_void_p(v.data_ptr()), C.c_void_p(t.data_ptr()),
           40, 100, 0.0, C.byref(sw), C.byref(dl), N.stream_handle())
    ref32 = op.jacobi_sweeps(rho, (nx, ny, nz), np.float32(h), 40, dtype=np.float32)
    got = v.cpu().numpy()
    assert sw.value == 40
    assert np.max(np.abs(got - ref32)) <= 1e-6 * np.max(np.abs(ref32))
    ref64 = op.jacobi_sweeps(rho, (nx, ny, nz), h, 40, dtype=np.float64)
    assert rel_l2(got, ref64) < 1e-5


def test_compute_hartree_iter_stops_at_cap(c0):
    sm, mol = c0
    g = _grid(sm, 16, 0.5)
    q = qmtools.QMTools.Compute_density(g, mol, precision="fp32")
    with pytest.warns(UserWarning):
        v = qmtools.QMTools.Compute_hartree_iter(q, mol, tolerance=1e-30, max_sweeps=400)
    assert v.sweeps == 400
